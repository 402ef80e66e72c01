// capi.cu -- the C ABI (include/dol_b200.h): argument checks, workspace
// handling, error reporting, and the one-call pipelines.
#include <float.h>
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "dol_b200.h"
#include "gen.cuh"
#include "kernels.h"

namespace dolk {
int g_num_sms = 148;
}

using namespace dolk;

namespace {

thread_local std::string t_err;

dol_status fail(dol_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return s;
}

// Per-device state: SM count and a mapped host word that kernels with bounded
// waits set when a wait gives up (read by dol_sync).  `ready` is published
// with release order after the other fields are written, so a thread that
// reads it true (acquire) also sees them.
struct DeviceState {
    std::atomic<bool> ready{false};
    int sms = 0;
    int* err_host = nullptr;
    int* err_dev = nullptr;
};
constexpr int kMaxDevices = 64;
DeviceState g_dev[kMaxDevices];
std::mutex g_init_mu;

dol_status device_state(DeviceState** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(DOL_ERR_UNSUPPORTED, "device index %d out of range", dev);
    DeviceState& s = g_dev[dev];
    if (!s.ready.load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(g_init_mu);
        if (!s.ready.load(std::memory_order_relaxed)) {
            int sms = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
            e = cudaHostAlloc(&s.err_host, sizeof(int), cudaHostAllocMapped);
            if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaHostAlloc: %s", cudaGetErrorString(e));
            *s.err_host = 0;
            e = cudaHostGetDevicePointer(&s.err_dev, s.err_host, 0);
            if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(e));
            // keep stream-ordered workspace allocations cached between calls
            // instead of returning them to the driver at every synchronisation
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
            s.sms = sms;
            s.ready.store(true, std::memory_order_release);
        }
    }
    g_num_sms = s.sms;
    *out = &s;
    return DOL_OK;
}

dol_status check_dims(int w, int h, int d)
{
    if (w < 1 || h < 1 || d < 1) return fail(DOL_ERR_INVALID_ARG, "dimensions must be >= 1 (got %d x %d x %d)", w, h, d);
    if ((long long)w * h * d > (1LL << 40)) return fail(DOL_ERR_INVALID_ARG, "volume too large");
    return DOL_OK;
}

dol_status check_cw(int cw)
{
    if (cw < 1 || cw > 64) return fail(DOL_ERR_INVALID_ARG, "cell width cw must be in [1, 64] (got %d)", cw);
    return DOL_OK;
}

dol_status launched(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return DOL_OK;
}

// Largest workspace the library allocates by itself (0: no limit); above it
// an entry point reports DOL_ERR_NO_MEMORY, Danielsson runs its serial engine.
std::atomic<size_t> g_workspace_limit{0};
// which Danielsson engine this thread's last call queued (dol_last_engine)
thread_local int t_engine = 0;

// Workspace: the caller's, or a stream-ordered allocation freed after the work.
struct Workspace {
    void* ptr = nullptr;
    bool owned = false;
    cudaStream_t st = nullptr;
    ~Workspace()
    {
        if (owned && ptr) cudaFreeAsync(ptr, st);
    }
};

dol_status get_workspace(Workspace& ws, void* user, size_t user_bytes, size_t need, cudaStream_t st)
{
    ws.st = st;
    if (need == 0) return DOL_OK;
    if (user) {
        if (user_bytes < need)
            return fail(DOL_ERR_INVALID_ARG, "workspace too small: %zu bytes given, %zu needed", user_bytes, need);
        dol_status s = (dol_status)check_dev_ptr(user, "workspace");
        if (s != DOL_OK) return s;
        ws.ptr = user;
        return DOL_OK;
    }
    const size_t cap = g_workspace_limit.load(std::memory_order_relaxed);
    if (cap && need > cap)
        return fail(DOL_ERR_NO_MEMORY, "workspace of %zu bytes exceeds the limit of %zu set by dol_set_workspace_limit",
                    need, cap);
    cudaError_t e = cudaMallocAsync(&ws.ptr, need, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DOL_ERR_NO_MEMORY, "workspace allocation of %zu bytes failed: %s", need, cudaGetErrorString(e));
    }
    ws.owned = true;
    return DOL_OK;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

// widest row the single-CTA sweeps handle (8 cells per thread, 512 threads),
// and the 3D FastSweep wavefront (8 cells per thread, 256 threads)
constexpr int kMaxSweepWidth = 4096;
constexpr int kMaxSweepWidth3 = 2048;

dol_status check_sweep_width(int w)
{
    if (w > kMaxSweepWidth)
        return fail(DOL_ERR_UNSUPPORTED, "row width %d exceeds the sweep kernels' limit of %d", w, kMaxSweepWidth);
    return DOL_OK;
}

#define DOL_TRY(x)                          \
    do {                                    \
        dol_status _s = (dol_status)(x);    \
        if (_s != DOL_OK) return _s;        \
    } while (0)

}  // namespace

int dolk::set_error(int s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return s;
}

// A pointer the GPU can dereference: device, managed, or mapped host memory.
int dolk::check_dev_ptr(const void* p, const char* name)
{
    if (!p) return fail(DOL_ERR_INVALID_ARG, "%s is NULL", name);
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DOL_ERR_INVALID_ARG, "%s is not a device pointer (%s)", name, cudaGetErrorString(e));
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return DOL_OK;
    if (a.type == cudaMemoryTypeHost && a.devicePointer == p) return DOL_OK;
    return fail(DOL_ERR_INVALID_ARG, "%s is not device-accessible memory", name);
}

extern "C" {

int dol_version(void) { return DOL_B200_VERSION; }

const char* dol_status_string(dol_status s)
{
    switch (s) {
        case DOL_OK: return "ok";
        case DOL_ERR_INVALID_ARG: return "invalid argument";
        case DOL_ERR_CUDA: return "CUDA error";
        case DOL_ERR_NO_MEMORY: return "out of device memory";
        case DOL_ERR_TIMEOUT: return "device-side wait timed out";
        case DOL_ERR_UNSUPPORTED: return "unsupported size or option";
    }
    return "unknown status";
}

const char* dol_last_error(void) { return t_err.c_str(); }

dol_status dol_sync(void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    cudaError_t e = cudaStreamSynchronize(S(stream));
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaStreamSynchronize: %s", cudaGetErrorString(e));
    if (*(volatile int*)ds->err_host) {
        *(volatile int*)ds->err_host = 0;
        return fail(DOL_ERR_TIMEOUT, "a bounded device-side wait gave up; results of that call are invalid");
    }
    return DOL_OK;
}

size_t dol_mask_words(int w, int h, int d)
{
    if (w < 1 || h < 1 || d < 1) return 0;
    return (size_t)((w + 31) / 32) * h * d;
}

// ---- host test-mask generators (the reference's own LCG and shapes) ---------------

void dol_add_points_2d(int w, int h, int n, uint32_t seed, uint32_t* mask)
{
    const int ws = (w + 31) / 32;
    for (int i = 0; i < n; i++) {
        seed = lcg_next(seed);
        int x = lcg_scale(seed, w);
        seed = lcg_next(seed);
        int y = lcg_scale(seed, h);
        mask[(size_t)y * ws + (x >> 5)] |= 1u << (x & 31);
    }
}

void dol_add_points_3d(int w, int h, int d, int n, uint32_t seed, uint32_t* mask)
{
    const int ws = (w + 31) / 32;
    for (int i = 0; i < n; i++) {
        seed = lcg_next(seed);
        int x = lcg_scale(seed, w);
        seed = lcg_next(seed);
        int y = lcg_scale(seed, h);
        seed = lcg_next(seed);
        int z = lcg_scale(seed, d);
        mask[((size_t)z * h + y) * ws + (x >> 5)] |= 1u << (x & 31);
    }
}

static void fill_cells(int ws, int x0, int x1, int y0, int y1, uint32_t* slice)
{
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++) slice[(size_t)y * ws + (x >> 5)] |= 1u << (x & 31);
}

void dol_add_block_2d(int w, int h, int sides, uint32_t* mask)
{
    const int ws = (w + 31) / 32;
    const int x0 = w / 4, x1 = x0 + w / 2 - 1, y0 = h / 3, y1 = y0 + h / 3 - 1;
    if (sides > 4) { fill_cells(ws, x0, x1, y0, y1, mask); return; }
    if (sides > 0) fill_cells(ws, x0, x1, y0, y0, mask);
    if (sides > 1) fill_cells(ws, x0, x0, y0, y1, mask);
    if (sides > 2) fill_cells(ws, x0, x1, y1, y1, mask);
    if (sides > 3) fill_cells(ws, x1, x1, y0, y1, mask);
}

void dol_add_block_3d(int w, int h, int d, int sides, uint32_t* mask)
{
    const int ws = (w + 31) / 32;
    const int x0 = w / 4, x1 = x0 + w / 2 - 1, y0 = h / 3, y1 = y0 + h / 3 - 1, z0 = d / 3, z1 = z0 + d / 3 - 1;
    auto box = [&](int a0, int a1, int b0, int b1, int c0, int c1) {
        for (int z = c0; z <= c1; z++) fill_cells(ws, a0, a1, b0, b1, mask + (size_t)z * ws * h);
    };
    if (sides > 6) { box(x0, x1, y0, y1, z0, z1); return; }
    if (sides > 0) box(x0, x1, y0, y1, z0, z0);
    if (sides > 1) box(x0, x0, y0, y1, z0, z1);
    if (sides > 2) box(x0, x1, y0, y0, z0, z1);
    if (sides > 3) box(x1, x1, y0, y1, z0, z1);
    if (sides > 4) box(x0, x1, y1, y1, z0, z1);
    if (sides > 5) box(x0, x1, y0, y1, z1, z1);
}

// ---- byte mask -> bitmask ---------------------------------------------------------------

dol_status dol_pack_bytemask(int w, int h, int d, const uint8_t* bytes, int threshold, int less_than, uint32_t* mask,
                             void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(bytes, "bytes"));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    launch_pack_bytemask(bytes, mask, w, (long long)h * d, threshold, less_than, S(stream));
    return launched("pack_bytemask");
}

// ---- initialisation -------------------------------------------------------------------

dol_status dol_init_distances_2d_i16(int w, int h, const uint32_t* mask, int16_t* dist, int16_t max_d, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    launch_init_distances_int<int16_t>(mask, dist, w, h, max_d, S(stream));
    return launched("init_distances_2d_i16");
}

dol_status dol_init_distances_2d_i32(int w, int h, const uint32_t* mask, int32_t* dist, int32_t max_d, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    launch_init_distances_int<int32_t>(mask, dist, w, h, max_d, S(stream));
    return launched("init_distances_2d_i32");
}

static dol_status chamfer_common(int w, int h, void* dist, bool wide, int* multiplier, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    if (w < 2) return fail(DOL_ERR_UNSUPPORTED, "Chamfer needs rows of at least 2 cells (the reference reads outside a 1-cell row)");
    DOL_TRY(check_sweep_width(w));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    if (wide)
        launch_chamfer_2d<int32_t>(static_cast<int32_t*>(dist), w, h, S(stream));
    else
        launch_chamfer_2d<int16_t>(static_cast<int16_t*>(dist), w, h, S(stream));
    if (multiplier) *multiplier = 3;
    return launched(wide ? "chamfer_2d_i32" : "chamfer_2d_i16");
}

dol_status dol_chamfer_2d_i16(int w, int h, int16_t* dist, int* multiplier, void* stream)
{
    return chamfer_common(w, h, dist, false, multiplier, stream);
}

dol_status dol_chamfer_2d_i32(int w, int h, int32_t* dist, int* multiplier, void* stream)
{
    return chamfer_common(w, h, dist, true, multiplier, stream);
}

dol_status dol_init_distances_2d(int w, int h, const uint32_t* mask, float* dist, float max_d, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    launch_init_distances(mask, dist, w, h, max_d, S(stream));
    return launched("init_distances_2d");
}

dol_status dol_init_deltas_2d(int w, int h, const uint32_t* mask, dol_delta2* deltas, int invert, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    launch_init_deltas(2, mask, deltas, w, h, invert, S(stream));
    return launched("init_deltas_2d");
}

dol_status dol_init_deltas_3d(int w, int h, int d, const uint32_t* mask, dol_delta3* deltas, int invert, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    launch_init_deltas(3, mask, deltas, w, (long long)h * d, invert, S(stream));
    return launched("init_deltas_3d");
}

dol_status dol_init_border_2d(int w, int h, const uint32_t* mask, dol_delta2* deltas, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    launch_init_border(2, mask, deltas, w, h, 1, S(stream));
    return launched("init_border_2d");
}

dol_status dol_init_border_3d(int w, int h, int d, const uint32_t* mask, dol_delta3* deltas, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    launch_init_border(3, mask, deltas, w, h, d, S(stream));
    return launched("init_border_3d");
}

// ---- propagation -------------------------------------------------------------------------

// The Danielsson entries: the block schedule on the caller's workspace or
// one the library allocates; without one (the allocation failed, or it is
// above the dol_set_workspace_limit cap), the serial engine, which needs no
// workspace but is much slower on large fields -- dol_last_engine() and
// dol_last_error() say so.
static dol_status danielsson_common(int dim, int w, int h, int d, void* deltas, int cw, void* workspace,
                                    size_t workspace_bytes, bool caller_ws, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_sweep_width(w));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    const int dd = dim == 3 ? d : 1;
    const size_t need = danielsson_workspace_bytes(dim, w, h, dd);
    Workspace ws;
    std::string why;
    if (caller_ws && workspace) {
        DOL_TRY(get_workspace(ws, workspace, workspace_bytes, need, S(stream)));
    } else if (need && get_workspace(ws, nullptr, 0, need, S(stream)) != DOL_OK) {
        why = t_err;   // the failed allocation's message
        ws.ptr = nullptr;
    }
    const bool blocks = run_danielsson(dim, deltas, w, h, dd, cw, ws.ptr, need, ds->err_dev, S(stream));
    t_engine = blocks ? DOL_ENGINE_BLOCKS : DOL_ENGINE_SERIAL;
    dol_status st = launched(dim == 3 ? "danielsson_3d" : "danielsson_2d");
    if (st == DOL_OK)
        t_err = blocks ? std::string()
                       : (need ? "danielsson: serial engine (no workspace for the block schedule: " +
                                     (why.empty() ? std::string("none given") : why) + ")"
                               : "danielsson: serial engine (the block schedule does not apply to this shape)");
    return st;
}

size_t dol_danielsson_workspace_size(int w, int h, int d)
{
    if (w < 1 || h < 1 || d < 1) return 0;
    return danielsson_workspace_bytes(d > 1 ? 3 : 2, w, h, d);
}

dol_status dol_danielsson_2d(int w, int h, dol_delta2* deltas, int cw, void* stream)
{
    return danielsson_common(2, w, h, 1, deltas, cw, nullptr, 0, false, stream);
}

dol_status dol_danielsson_3d(int w, int h, int d, dol_delta3* deltas, int cw, void* stream)
{
    return danielsson_common(3, w, h, d, deltas, cw, nullptr, 0, false, stream);
}

dol_status dol_danielsson_2d_ws(int w, int h, dol_delta2* deltas, int cw, void* workspace, size_t workspace_bytes,
                                void* stream)
{
    return danielsson_common(2, w, h, 1, deltas, cw, workspace, workspace_bytes, true, stream);
}

dol_status dol_danielsson_3d_ws(int w, int h, int d, dol_delta3* deltas, int cw, void* workspace,
                                size_t workspace_bytes, void* stream)
{
    return danielsson_common(3, w, h, d, deltas, cw, workspace, workspace_bytes, true, stream);
}

int dol_last_engine(void) { return t_engine; }

void dol_set_workspace_limit(size_t bytes) { g_workspace_limit.store(bytes, std::memory_order_relaxed); }

dol_status dol_fastsweep_2d(int w, int h, dol_delta2* deltas, int cw, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_sweep_width(w));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    launch_fastsweep_2d(deltas, w, h, cw, S(stream));
    return launched("fastsweep_2d");
}

size_t dol_fastsweep_3d_workspace_size(int w, int h, int d) { return fastsweep3_workspace_bytes(w, h, d); }

dol_status dol_fastsweep_3d(int w, int h, int d, dol_delta3* deltas, int cw, void* workspace, size_t workspace_bytes,
                            void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_sweep_width(w));
    if (w > kMaxSweepWidth3) return fail(DOL_ERR_UNSUPPORTED, "3D FastSweep rows are limited to %d cells", kMaxSweepWidth3);
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, fastsweep3_workspace_bytes(w, h, d), S(stream)));
    launch_fastsweep_3d(deltas, w, h, d, cw, ws.ptr, ds->err_dev, S(stream));
    return launched("fastsweep_3d");
}

size_t dol_jumpflood_2d_workspace_size(int w, int h) { return jumpflood_workspace_bytes(2, w, h, 1); }
size_t dol_jumpflood_3d_workspace_size(int w, int h, int d) { return jumpflood_workspace_bytes(3, w, h, d); }

dol_status dol_jumpflood_2d(int w, int h, dol_delta2* deltas, int cw, void* workspace, size_t workspace_bytes,
                            void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_jumpflood_2d_workspace_size(w, h), S(stream)));
    launch_jumpflood(2, deltas, ws.ptr, w, h, 1, cw, S(stream));
    return launched("jumpflood_2d");
}

dol_status dol_jumpflood_3d(int w, int h, int d, dol_delta3* deltas, int cw, void* workspace, size_t workspace_bytes,
                            void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_cw(cw));
    if (d > 65535) return fail(DOL_ERR_UNSUPPORTED, "JumpFlood volumes are limited to 65535 slices");
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_jumpflood_3d_workspace_size(w, h, d), S(stream)));
    launch_jumpflood(3, deltas, ws.ptr, w, h, d, cw, S(stream));
    return launched("jumpflood_3d");
}

// ---- Felzenszwalb ----------------------------------------------------------------------------

size_t dol_felzenszwalb_2d_workspace_size(int w, int h) { return felz_float_workspace_bytes(w, h); }

dol_status dol_felzenszwalb_2d(int w, int h, float* dist, void* workspace, size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, felz_float_workspace_bytes(w, h), S(stream)));
    launch_felz_float_2d(dist, w, h, ws.ptr, S(stream));
    return launched("felzenszwalb_2d");
}

size_t dol_edt_mask_2d_workspace_size(int w, int h) { return edt_workspace_bytes(2, w, h, 1); }
size_t dol_edt_mask_3d_workspace_size(int w, int h, int d) { return edt_workspace_bytes(3, w, h, d); }

static dol_status edt_common(int dim, int w, int h, int d, const uint32_t* mask, float* out, int form, void* workspace,
                             size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    if (form != DOL_EDT_SQUARED && form != DOL_EDT_DIST && form != DOL_EDT_SIGNED)
        return fail(DOL_ERR_INVALID_ARG, "form must be DOL_EDT_SQUARED, DOL_EDT_DIST or DOL_EDT_SIGNED");
    if (w > 16384 || h > 16384 || d > 16384) return fail(DOL_ERR_UNSUPPORTED, "EDT dimensions are limited to 16384");
    if (h > 65535 || d > 65535) return fail(DOL_ERR_UNSUPPORTED, "EDT grid limit");
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(out, "out"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, edt_workspace_bytes(dim, w, h, d), S(stream)));
    launch_edt_mask(dim, mask, out, w, h, d, form, ws.ptr, ds->err_dev, S(stream));
    return launched("edt_mask");
}

dol_status dol_edt_mask_2d(int w, int h, const uint32_t* mask, float* out, int form, void* workspace,
                           size_t workspace_bytes, void* stream)
{
    return edt_common(2, w, h, 1, mask, out, form, workspace, workspace_bytes, stream);
}

dol_status dol_edt_mask_3d(int w, int h, int d, const uint32_t* mask, float* out, int form, void* workspace,
                           size_t workspace_bytes, void* stream)
{
    return edt_common(3, w, h, d, mask, out, form, workspace, workspace_bytes, stream);
}

// ---- deltas -> distances -------------------------------------------------------------------------

dol_status dol_deltas_to_dist_2d(int w, int h, const dol_delta2* deltas, int cw, const uint32_t* sign_mask, float* out,
                                 void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    DOL_TRY(check_dev_ptr(out, "out"));
    if (sign_mask) DOL_TRY(check_dev_ptr(sign_mask, "sign_mask"));
    launch_deltas_to_dist(2, deltas, cw, sign_mask, out, w, h, 1, S(stream));
    return launched("deltas_to_dist_2d");
}

dol_status dol_deltas_to_dist_3d(int w, int h, int d, const dol_delta3* deltas, int cw, const uint32_t* sign_mask,
                                 float* out, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_cw(cw));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    DOL_TRY(check_dev_ptr(out, "out"));
    if (sign_mask) DOL_TRY(check_dev_ptr(sign_mask, "sign_mask"));
    launch_deltas_to_dist(3, deltas, cw, sign_mask, out, w, h, d, S(stream));
    return launched("deltas_to_dist_3d");
}

// ---- occlusion ----------------------------------------------------------------------------------

static dol_status occ_checks(int w, int h, int d)
{
    DOL_TRY(check_dims(w, h, d));
    if ((long long)d * h > (1LL << 40) / 8) return fail(DOL_ERR_INVALID_ARG, "volume too large");
    return DOL_OK;
}

dol_status dol_init_dirw_2d(int w, int h, const uint32_t* mask, float* dirW, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, 1));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(dirW, "dirW"));
    launch_init_dirw(2, mask, dirW, w, h, 1, S(stream));
    return launched("init_dirw_2d");
}

dol_status dol_init_dirw_3d(int w, int h, int d, const uint32_t* mask, float* dirW, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(dirW, "dirW"));
    launch_init_dirw(3, mask, dirW, w, h, d, S(stream));
    return launched("init_dirw_3d");
}

dol_status dol_occlusion_sweep_2d(int w, int h, float* dirW, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(occ_checks(w, h, 1));
    DOL_TRY(check_dev_ptr(dirW, "dirW"));
    launch_occlusion_sweep(2, dirW, nullptr, w, h, 1, S(stream));
    return launched("occlusion_sweep_2d");
}

dol_status dol_occlusion_sweep_3d(int w, int h, int d, float* dirW, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(occ_checks(w, h, d));
    DOL_TRY(check_dev_ptr(dirW, "dirW"));
    launch_occlusion_sweep(3, dirW, nullptr, w, h, d, S(stream));
    return launched("occlusion_sweep_3d");
}

dol_status dol_occlusion_sweep_3d_io(int w, int h, int d, const float* in, float* out, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(occ_checks(w, h, d));
    DOL_TRY(check_dev_ptr(in, "in"));
    DOL_TRY(check_dev_ptr(out, "out"));
    if (in == out) return fail(DOL_ERR_INVALID_ARG, "the in/out occlusion sweep needs distinct in and out fields");
    launch_occlusion_sweep(3, out, in, w, h, d, S(stream));
    return launched("occlusion_sweep_3d_io");
}

// ---- mesh voxeliser -------------------------------------------------------------------------------

dol_status dol_voxelize_triangles(int tri_count, const int* indices, const float* vertices, const float* bbox, int w,
                                  int h, int d, uint32_t* mask, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    if (tri_count < 0) return fail(DOL_ERR_INVALID_ARG, "negative triangle count");
    if (!bbox) return fail(DOL_ERR_INVALID_ARG, "bbox is NULL");
    for (int i = 0; i < 3; i++)
        if (!(bbox[3 + i] > bbox[i]))   // also rejects NaN
            return fail(DOL_ERR_INVALID_ARG, "bbox extent %d is not positive (%g .. %g)", i, bbox[i], bbox[3 + i]);
    DOL_TRY(check_dev_ptr(mask, "mask"));
    if (tri_count > 0) {
        DOL_TRY(check_dev_ptr(vertices, "vertices"));
        if (indices) DOL_TRY(check_dev_ptr(indices, "indices"));
    }
    launch_voxelize(tri_count, indices, vertices, bbox, w, h, d, mask, S(stream));
    return launched("voxelize_triangles");
}

// ---- one-call signed fields ----------------------------------------------------------------------

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t dol_sdf_workspace_size(int w, int h, int d, int method)
{
    const int dim = d > 1 ? 3 : 2;
    const size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    const size_t cb = dim == 3 ? sizeof(dol_delta3) : sizeof(dol_delta2);
    if (method == DOL_FELZENSZWALB) return edt_workspace_bytes(dim, w, h, d);
    size_t b = align256(cells * cb);                       // deltas, when the caller passes none
    if (method == DOL_JUMPFLOOD) b += align256(jumpflood_workspace_bytes(dim, w, h, dim == 3 ? d : 1));
    if (method == DOL_FASTSWEEP && dim == 3) b += align256(fastsweep3_workspace_bytes(w, h, d));
    if (method == DOL_DANIELSSON) b += align256(danielsson_workspace_bytes(dim, w, h, dim == 3 ? d : 1));
    return b;
}

static dol_status sdf_common(int dim, int w, int h, int d, const uint32_t* mask, int method, void* deltas, float* dist,
                             void* workspace, size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    if (deltas) DOL_TRY(check_dev_ptr(deltas, "deltas"));
    if (dist) DOL_TRY(check_dev_ptr(dist, "dist"));
    if (!deltas && !dist) return fail(DOL_ERR_INVALID_ARG, "at least one of deltas / dist is required");
    if (method != DOL_DANIELSSON && method != DOL_FASTSWEEP && method != DOL_JUMPFLOOD && method != DOL_FELZENSZWALB)
        return fail(DOL_ERR_INVALID_ARG, "unknown method %d", method);
    if (method == DOL_FELZENSZWALB && deltas)
        return fail(DOL_ERR_INVALID_ARG, "Felzenszwalb produces distances only; pass deltas = NULL");
    if (method == DOL_DANIELSSON || method == DOL_FASTSWEEP) DOL_TRY(check_sweep_width(w));
    if (method == DOL_FASTSWEEP && dim == 3 && w > kMaxSweepWidth3)
        return fail(DOL_ERR_UNSUPPORTED, "3D FastSweep rows are limited to %d cells", kMaxSweepWidth3);
    if (method == DOL_JUMPFLOOD && dim == 3 && d > 65535)
        return fail(DOL_ERR_UNSUPPORTED, "JumpFlood volumes are limited to 65535 slices");
    cudaStream_t st = S(stream);
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_sdf_workspace_size(w, h, dim == 3 ? d : 1, method), st));

    if (method == DOL_FELZENSZWALB) {
        launch_edt_mask(dim, mask, dist, w, h, d, DOL_EDT_SIGNED, ws.ptr, ds->err_dev, st);
        return launched("sdf (felzenszwalb)");
    }
    const size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    const size_t cb = dim == 3 ? sizeof(dol_delta3) : sizeof(dol_delta2);
    char* p = static_cast<char*>(ws.ptr);
    void* dl = deltas ? deltas : p;
    p += align256(cells * cb);
    launch_init_border(dim, mask, dl, w, h, d, st);
    if (method == DOL_DANIELSSON) {
        run_danielsson(dim, dl, w, h, d, 2, p, danielsson_workspace_bytes(dim, w, h, dim == 3 ? d : 1), ds->err_dev,
                       st);
    } else if (method == DOL_FASTSWEEP) {
        if (dim == 2)
            launch_fastsweep_2d(dl, w, h, 2, st);
        else
            launch_fastsweep_3d(dl, w, h, d, 2, p, ds->err_dev, st);
    } else {
        launch_jumpflood(dim, dl, p, w, h, d, 2, st);
    }
    if (dist) launch_deltas_to_dist(dim, dl, 2, mask, dist, w, h, d, st);
    return launched("sdf");
}

dol_status dol_sdf_2d(int w, int h, const uint32_t* mask, int method, dol_delta2* deltas, float* dist, void* workspace,
                      size_t workspace_bytes, void* stream)
{
    return sdf_common(2, w, h, 1, mask, method, deltas, dist, workspace, workspace_bytes, stream);
}

dol_status dol_sdf_3d(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* deltas, float* dist,
                      void* workspace, size_t workspace_bytes, void* stream)
{
    return sdf_common(3, w, h, d, mask, method, deltas, dist, workspace, workspace_bytes, stream);
}

// ---- two-pass signed fields (the tool's -S path) --------------------------------------------------

size_t dol_sdf_two_pass_workspace_size(int w, int h, int d, int method)
{
    const int dim = d > 1 ? 3 : 2;
    const size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    const size_t cb = dim == 3 ? sizeof(dol_delta3) : sizeof(dol_delta2);
    size_t b = 2 * align256(cells * cb);                    // exterior / interior deltas the caller does not keep
    if (method == DOL_JUMPFLOOD) b += align256(jumpflood_workspace_bytes(dim, w, h, dim == 3 ? d : 1));
    if (method == DOL_FASTSWEEP && dim == 3) b += align256(fastsweep3_workspace_bytes(w, h, d));
    if (method == DOL_DANIELSSON) b += align256(danielsson_workspace_bytes(dim, w, h, dim == 3 ? d : 1));
    return b;
}

static dol_status sdf_two_pass_common(int dim, int w, int h, int d, const uint32_t* mask, int method, void* ext,
                                      void* intr, float* dist, void* workspace, size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    if (ext) DOL_TRY(check_dev_ptr(ext, "exterior"));
    if (intr) DOL_TRY(check_dev_ptr(intr, "interior"));
    if (dist) DOL_TRY(check_dev_ptr(dist, "dist"));
    if (!ext && !intr && !dist) return fail(DOL_ERR_INVALID_ARG, "at least one of exterior / interior / dist is required");
    if (method != DOL_DANIELSSON && method != DOL_FASTSWEEP && method != DOL_JUMPFLOOD)
        return fail(DOL_ERR_INVALID_ARG, "the two-pass field takes Danielsson, FastSweep or JumpFlood, not method %d",
                    method);
    if (method == DOL_DANIELSSON || method == DOL_FASTSWEEP) DOL_TRY(check_sweep_width(w));
    if (method == DOL_FASTSWEEP && dim == 3 && w > kMaxSweepWidth3)
        return fail(DOL_ERR_UNSUPPORTED, "3D FastSweep rows are limited to %d cells", kMaxSweepWidth3);
    if (method == DOL_JUMPFLOOD && dim == 3 && d > 65535)
        return fail(DOL_ERR_UNSUPPORTED, "JumpFlood volumes are limited to 65535 slices");
    cudaStream_t st = S(stream);
    const int dd = dim == 3 ? d : 1;
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_sdf_two_pass_workspace_size(w, h, dd, method), st));
    const size_t cells = (size_t)w * h * dd;
    const size_t cb = dim == 3 ? sizeof(dol_delta3) : sizeof(dol_delta2);
    char* p = static_cast<char*>(ws.ptr);
    void* de = ext ? ext : p;
    p += align256(cells * cb);
    void* di = intr ? intr : p;
    p += align256(cells * cb);
    const long long rows = (long long)h * dd;
    launch_init_deltas(dim, mask, de, w, rows, 0, st);   // deltas to set cells
    launch_init_deltas(dim, mask, di, w, rows, 1, st);   // deltas to clear cells
    for (void* dl : {de, di}) {
        if (method == DOL_DANIELSSON) {
            run_danielsson(dim, dl, w, h, dd, 1, p, danielsson_workspace_bytes(dim, w, h, dd), ds->err_dev, st);
        } else if (method == DOL_FASTSWEEP) {
            if (dim == 2)
                launch_fastsweep_2d(dl, w, h, 1, st);
            else
                launch_fastsweep_3d(dl, w, h, d, 1, p, ds->err_dev, st);
        } else {
            launch_jumpflood(dim, dl, p, w, h, dd, 1, st);
        }
    }
    if (dist) launch_two_pass_dist(dim, de, di, dist, (long long)cells, st);
    return launched("sdf_two_pass");
}

dol_status dol_sdf_two_pass_2d(int w, int h, const uint32_t* mask, int method, dol_delta2* exterior,
                               dol_delta2* interior, float* dist, void* workspace, size_t workspace_bytes, void* stream)
{
    return sdf_two_pass_common(2, w, h, 1, mask, method, exterior, interior, dist, workspace, workspace_bytes, stream);
}

dol_status dol_sdf_two_pass_3d(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* exterior,
                               dol_delta3* interior, float* dist, void* workspace, size_t workspace_bytes, void* stream)
{
    return sdf_two_pass_common(3, w, h, d, mask, method, exterior, interior, dist, workspace, workspace_bytes, stream);
}

// ---- batched signed fields ------------------------------------------------------------------------

size_t dol_batch_workspace_size(int n)
{
    if (n < 1) return 0;
    return align256((size_t)n * sizeof(dol_batch_item)) + align256((size_t)n * sizeof(int)) + 256;
}

dol_status dol_batch_prepare(int n, const dol_batch_item* items, void* workspace, size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    if (n < 1 || !items) return fail(DOL_ERR_INVALID_ARG, "need at least one item");
    if (!workspace) return fail(DOL_ERR_INVALID_ARG, "dol_batch_prepare needs a workspace (dol_batch_workspace_size)");
    if (workspace_bytes < dol_batch_workspace_size(n)) return fail(DOL_ERR_INVALID_ARG, "workspace too small");
    DOL_TRY(check_dev_ptr(workspace, "workspace"));
    std::vector<int> order(n);
    std::vector<double> work(n);
    for (int i = 0; i < n; i++) {
        const dol_batch_item& it = items[i];
        if (it.w < 1 || it.h < 1 || it.d < 1) return fail(DOL_ERR_INVALID_ARG, "item %d has an empty size", i);
        if (it.w > 1024) return fail(DOL_ERR_UNSUPPORTED, "item %d: batched rows are limited to 1024 cells", i);
        if (it.mask_word_offset < 0 || it.delta_byte_offset < 0)
            return fail(DOL_ERR_INVALID_ARG, "item %d has a negative offset", i);
        // 2D cells are read and written as 4-byte words, 3D cells as 2-byte halves
        if (it.delta_byte_offset % (it.d > 1 ? 2 : 4) != 0)
            return fail(DOL_ERR_INVALID_ARG, "item %d: delta_byte_offset %lld is not a multiple of %d bytes", i,
                        it.delta_byte_offset, it.d > 1 ? 2 : 4);
        // serial row steps dominate: 2h per image, 2(d-1)*2h per volume, plus the cells themselves
        work[i] = it.d > 1 ? 4.0 * it.d * it.h + 1e-3 * it.w * it.h * it.d : 2.0 * it.h + 1e-3 * it.w * it.h;
        order[i] = i;
    }
    // queue A: volumes with rows of at most 256 cells (one warp each); queue B:
    // items with wider rows (one CTA each), then the narrow images; each group
    // by decreasing work
    auto group = [&](int i) { return items[i].w > 256 ? 1 : (items[i].d > 1 ? 0 : 2); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const int ga = group(a), gb = group(b);
        if (ga != gb) return ga < gb;
        return work[a] > work[b];
    });
    int nv = 0;
    for (int i = 0; i < n; i++) nv += group(i) == 0;
    char* p = static_cast<char*>(workspace);
    cudaStream_t st = S(stream);
    cudaError_t e = cudaMemcpyAsync(p, items, (size_t)n * sizeof(dol_batch_item), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p + align256((size_t)n * sizeof(dol_batch_item)), order.data(), (size_t)n * sizeof(int),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p + align256((size_t)n * sizeof(dol_batch_item)) + align256((size_t)n * sizeof(int)) +
                                2 * sizeof(int),
                            &nv, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // the host order vector ends here
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "batch upload: %s", cudaGetErrorString(e));
    return DOL_OK;
}

dol_status dol_batch_run(int n, const uint32_t* masks, void* deltas, float* dist, void* workspace, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    if (n < 1 || !masks || !deltas || !workspace) return fail(DOL_ERR_INVALID_ARG, "missing batch buffer");
    if (((uintptr_t)masks | (uintptr_t)deltas | (uintptr_t)dist) % 4 != 0)
        return fail(DOL_ERR_INVALID_ARG, "batch buffers must be 4-byte aligned");
    char* p = static_cast<char*>(workspace);
    const void* items = p;
    const int* order = reinterpret_cast<const int*>(p + align256((size_t)n * sizeof(dol_batch_item)));
    int* counter = reinterpret_cast<int*>(p + align256((size_t)n * sizeof(dol_batch_item)) +
                                          align256((size_t)n * sizeof(int)));
    launch_batch_sdf(items, order, n, masks, deltas, dist, counter, S(stream));
    return launched("batch_sdf");
}

dol_status dol_batch_sdf(int n, const dol_batch_item* items, const uint32_t* masks, void* deltas, float* dist,
                         void* workspace, size_t workspace_bytes, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dev_ptr(masks, "masks"));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    if (dist) DOL_TRY(check_dev_ptr(dist, "dist"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_batch_workspace_size(n), S(stream)));
    DOL_TRY(dol_batch_prepare(n, items, ws.ptr, dol_batch_workspace_size(n), stream));
    return dol_batch_run(n, masks, deltas, dist, ws.ptr, stream);
}

namespace {
struct GraphHandle {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};
}  // namespace

dol_status dol_batch_graph_create(int n, const uint32_t* masks, void* deltas, float* dist, void* workspace, void** out)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    if (!out) return fail(DOL_ERR_INVALID_ARG, "graph output pointer is NULL");
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail(DOL_ERR_CUDA, "stream");
    GraphHandle* g = new GraphHandle;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    dol_status s = DOL_OK;
    if (e == cudaSuccess) {
        s = dol_batch_run(n, masks, deltas, dist, workspace, st);
        e = cudaStreamEndCapture(st, &g->graph);
    }
    if (e == cudaSuccess && s == DOL_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    cudaStreamDestroy(st);
    if (e != cudaSuccess || s != DOL_OK) {
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        cudaGetLastError();
        return s != DOL_OK ? s : fail(DOL_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    }
    *out = g;
    return DOL_OK;
}

dol_status dol_graph_launch(void* graph, void* stream)
{
    if (!graph) return fail(DOL_ERR_INVALID_ARG, "graph is NULL");
    cudaError_t e = cudaGraphLaunch(static_cast<GraphHandle*>(graph)->exec, S(stream));
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(e));
    return DOL_OK;
}

void dol_graph_destroy(void* graph)
{
    GraphHandle* g = static_cast<GraphHandle*>(graph);
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

// ---- float sites ---------------------------------------------------------------------------------

static dol_status sites_common(int dim, int w, int h, int d, int n)
{
    if (dim != 2 && dim != 3) return fail(DOL_ERR_INVALID_ARG, "dim must be 2 or 3");
    if (dim == 2 && d != 1) return fail(DOL_ERR_INVALID_ARG, "2D site grids have d = 1");
    DOL_TRY(check_dims(w, h, d));
    if (n < 0) return fail(DOL_ERR_INVALID_ARG, "negative site count");
    return DOL_OK;
}

dol_status dol_sites_seed(int dim, int w, int h, int d, int n, const float* sites, uint32_t* mask, int* cell_site,
                          void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(sites_common(dim, w, h, d, n));
    if (n > 0) DOL_TRY(check_dev_ptr(sites, "sites"));
    DOL_TRY(check_dev_ptr(mask, "mask"));
    DOL_TRY(check_dev_ptr(cell_site, "cell_site"));
    launch_sites_seed(dim, w, h, d, n, sites, mask, cell_site, S(stream));
    return launched("sites_seed");
}

dol_status dol_sites_forward(int dim, int w, int h, int d, int n, const void* deltas, const int* cell_site,
                             const float* sites, int* owner, float* dist, void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(sites_common(dim, w, h, d, n));
    DOL_TRY(check_dev_ptr(deltas, "deltas"));
    DOL_TRY(check_dev_ptr(cell_site, "cell_site"));
    if (n > 0) DOL_TRY(check_dev_ptr(sites, "sites"));
    DOL_TRY(check_dev_ptr(owner, "owner"));
    DOL_TRY(check_dev_ptr(dist, "dist"));
    launch_sites_forward(dim, w, h, d, n, deltas, cell_site, sites, owner, dist, S(stream));
    return launched("sites_forward");
}

size_t dol_sites_backward_workspace_size(int dim, int n) { return n > 0 ? (size_t)n * dim * sizeof(double) : 0; }

dol_status dol_sites_backward(int dim, int w, int h, int d, int n, const int* owner, const float* sites,
                              const float* grad_dist, float* grad_sites, void* workspace, size_t workspace_bytes,
                              void* stream)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(sites_common(dim, w, h, d, n));
    if (n == 0) return DOL_OK;
    DOL_TRY(check_dev_ptr(owner, "owner"));
    DOL_TRY(check_dev_ptr(sites, "sites"));
    DOL_TRY(check_dev_ptr(grad_dist, "grad_dist"));
    DOL_TRY(check_dev_ptr(grad_sites, "grad_sites"));
    Workspace ws;
    DOL_TRY(get_workspace(ws, workspace, workspace_bytes, dol_sites_backward_workspace_size(dim, n), S(stream)));
    launch_sites_backward(dim, w, h, d, n, owner, sites, grad_dist, static_cast<double*>(ws.ptr), grad_sites,
                          S(stream));
    return launched("sites_backward");
}

// ---- host-buffer variants --------------------------------------------------------------------------

namespace {
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf()
    {
        if (p) cudaFreeAsync(p, st);
    }
    dol_status alloc(size_t n, cudaStream_t s)
    {
        st = s;
        if (n == 0) return DOL_OK;
        cudaError_t e = cudaMallocAsync(&p, n, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(DOL_ERR_NO_MEMORY, "device allocation of %zu bytes failed", n);
        }
        return DOL_OK;
    }
};

struct OwnStream {
    cudaStream_t st = nullptr;
    ~OwnStream()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

dol_status copy(void* dst, const void* src, size_t n, cudaMemcpyKind k, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, n, k, st);
    if (e != cudaSuccess) return fail(DOL_ERR_CUDA, "cudaMemcpyAsync: %s", cudaGetErrorString(e));
    return DOL_OK;
}
}  // namespace

static dol_status sdf_host(int dim, int w, int h, int d, const uint32_t* mask, int method, void* deltas, float* dist)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    if (!mask) return fail(DOL_ERR_INVALID_ARG, "mask is NULL");
    if (!deltas && !dist) return fail(DOL_ERR_INVALID_ARG, "at least one of deltas / dist is required");
    OwnStream os;
    if (cudaStreamCreateWithFlags(&os.st, cudaStreamNonBlocking) != cudaSuccess)
        return fail(DOL_ERR_CUDA, "cudaStreamCreate failed");
    const size_t cells = (size_t)w * h * d;
    const size_t cb = dim == 3 ? sizeof(dol_delta3) : sizeof(dol_delta2);
    const size_t mb = dol_mask_words(w, h, d) * sizeof(uint32_t);
    DevBuf dm, dd, df;
    DOL_TRY(dm.alloc(mb, os.st));
    if (deltas) DOL_TRY(dd.alloc(cells * cb, os.st));
    if (dist) DOL_TRY(df.alloc(cells * sizeof(float), os.st));
    DOL_TRY(copy(dm.p, mask, mb, cudaMemcpyHostToDevice, os.st));
    dol_status s = sdf_common(dim, w, h, d, static_cast<uint32_t*>(dm.p), method, dd.p, static_cast<float*>(df.p),
                              nullptr, 0, os.st);
    if (s != DOL_OK) return s;
    if (deltas) DOL_TRY(copy(deltas, dd.p, cells * cb, cudaMemcpyDeviceToHost, os.st));
    if (dist) DOL_TRY(copy(dist, df.p, cells * sizeof(float), cudaMemcpyDeviceToHost, os.st));
    return dol_sync(os.st);
}

dol_status dol_sdf_2d_host(int w, int h, const uint32_t* mask, int method, dol_delta2* deltas, float* dist)
{
    return sdf_host(2, w, h, 1, mask, method, deltas, dist);
}

dol_status dol_sdf_3d_host(int w, int h, int d, const uint32_t* mask, int method, dol_delta3* deltas, float* dist)
{
    return sdf_host(3, w, h, d, mask, method, deltas, dist);
}

// Host-buffer 3D EDT with the copies overlapped: the mask goes up in slabs of
// slices on the copy-in stream, the x and y passes of a slab start when its
// slices have arrived, and the z pass runs in chunks of y whose rows go back
// to the host on two copy-out streams in turn (cudaMemcpy2DAsync: the chunk's
// rows of every slice, one slice pitch apart) while the next chunk computes.
constexpr int kHostSlabs = 8, kHostChunks = 16;
struct HostCopies {
    const uint32_t* hmask;
    uint32_t* dmask;
    float* host;
    const float* dev;
    int w, h, d;
    cudaStream_t compute, in, out[2];
    cudaEvent_t ev[kHostSlabs + kHostChunks];
    int n;
    cudaError_t err;
};

static void slab_ready(void* ctx, int z0, int z1)
{
    HostCopies* hc = static_cast<HostCopies*>(ctx);
    if (hc->err != cudaSuccess || hc->n >= kHostSlabs + kHostChunks) return;
    const size_t words = (size_t)((hc->w + 31) / 32) * hc->h;   // mask words per slice
    cudaEvent_t e = hc->ev[hc->n++];
    cudaError_t r = cudaMemcpyAsync(hc->dmask + (size_t)z0 * words, hc->hmask + (size_t)z0 * words,
                                    (size_t)(z1 - z0) * words * sizeof(uint32_t), cudaMemcpyHostToDevice, hc->in);
    if (r == cudaSuccess) r = cudaEventRecord(e, hc->in);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(hc->compute, e, 0);
    if (r != cudaSuccess) hc->err = r;
}

static void chunk_done(void* ctx, int y0, int y1)
{
    HostCopies* hc = static_cast<HostCopies*>(ctx);
    if (hc->err != cudaSuccess || hc->n >= kHostSlabs + kHostChunks) return;
    const int i = hc->n;
    cudaEvent_t e = hc->ev[hc->n++];
    cudaStream_t cs = hc->out[i & 1];
    const size_t pitch = (size_t)hc->w * hc->h * sizeof(float);
    const size_t first = (size_t)y0 * hc->w;
    cudaError_t r = cudaEventRecord(e, hc->compute);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(cs, e, 0);
    if (r == cudaSuccess)
        r = cudaMemcpy2DAsync(hc->host + first, pitch, hc->dev + first, pitch, (size_t)(y1 - y0) * hc->w * sizeof(float),
                              (size_t)hc->d, cudaMemcpyDeviceToHost, cs);
    if (r != cudaSuccess) hc->err = r;
}

dol_status dol_edt_mask_3d_host(int w, int h, int d, const uint32_t* mask, float* out, int form)
{
    DeviceState* ds;
    DOL_TRY(device_state(&ds));
    DOL_TRY(check_dims(w, h, d));
    if (!mask || !out) return fail(DOL_ERR_INVALID_ARG, "mask and out are required");
    if (form != DOL_EDT_SQUARED && form != DOL_EDT_DIST && form != DOL_EDT_SIGNED)
        return fail(DOL_ERR_INVALID_ARG, "form must be DOL_EDT_SQUARED, DOL_EDT_DIST or DOL_EDT_SIGNED");
    if (w > 16384 || h > 16384 || d > 16384) return fail(DOL_ERR_UNSUPPORTED, "EDT dimensions are limited to 16384");
    OwnStream os, is, o0, o1;
    for (OwnStream* p : {&os, &is, &o0, &o1})
        if (cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking) != cudaSuccess)
            return fail(DOL_ERR_CUDA, "cudaStreamCreate failed");
    const size_t cells = (size_t)w * h * d;
    const size_t mb = dol_mask_words(w, h, d) * sizeof(uint32_t);
    DevBuf dm, df, dw;
    DOL_TRY(dm.alloc(mb, os.st));
    DOL_TRY(df.alloc(cells * sizeof(float), os.st));
    DOL_TRY(dw.alloc(edt_workspace_bytes(3, w, h, d), os.st));
    // the copy-in stream starts after the allocations it writes into
    cudaEvent_t start;
    if (cudaEventCreateWithFlags(&start, cudaEventDisableTiming) != cudaSuccess)
        return fail(DOL_ERR_CUDA, "cudaEventCreate failed");
    cudaEventRecord(start, os.st);
    cudaStreamWaitEvent(is.st, start, 0);
    cudaEventDestroy(start);
    HostCopies hc{mask, static_cast<uint32_t*>(dm.p), out, static_cast<const float*>(df.p), w, h, d,
                  os.st, is.st, {o0.st, o1.st}, {}, 0, cudaSuccess};
    const int nev = kHostSlabs + kHostChunks;
    for (int i = 0; i < nev; i++)
        if (cudaEventCreateWithFlags(&hc.ev[i], cudaEventDisableTiming) != cudaSuccess) {
            for (int j = 0; j < i; j++) cudaEventDestroy(hc.ev[j]);
            return fail(DOL_ERR_CUDA, "cudaEventCreate failed");
        }
    const int slabs = d >= 2 * kHostSlabs ? kHostSlabs : 1;
    const int chunks = h >= 8 * kHostChunks ? kHostChunks : (h >= 64 ? 8 : 1);
    launch_edt_mask_3d_chunked(static_cast<uint32_t*>(dm.p), static_cast<float*>(df.p), w, h, d, form, dw.p,
                               ds->err_dev, os.st, slabs, slab_ready, chunks, chunk_done, &hc);
    const cudaError_t le = cudaGetLastError();
    // the copies back must finish before the device buffers are released (the
    // DevBuf destructors free on the compute stream)
    for (cudaStream_t cs : {o0.st, o1.st}) {
        cudaEvent_t fin;
        if (cudaEventCreateWithFlags(&fin, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(fin, cs);
            cudaStreamWaitEvent(os.st, fin, 0);
            cudaEventDestroy(fin);
        } else {
            cudaStreamSynchronize(cs);
        }
    }
    for (int i = 0; i < nev; i++) cudaEventDestroy(hc.ev[i]);
    if (le != cudaSuccess) return fail(DOL_ERR_CUDA, "launch failed: %s", cudaGetErrorString(le));
    if (hc.err != cudaSuccess) return fail(DOL_ERR_CUDA, "host copy failed: %s", cudaGetErrorString(hc.err));
    dol_status st = DOL_OK;
    for (cudaStream_t cs : {is.st, o0.st, o1.st, os.st}) {
        const dol_status si = dol_sync(cs);
        if (st == DOL_OK) st = si;
    }
    return st;
}

}  // extern "C"
