// k_edt_noalloc.cu -- the 2D mask-driven EDT for callers that cannot allocate.
//
// dol_edt_mask_2d needs w*h uint16 of scratch; by default it takes it from the
// caller's workspace or allocates it stream-ordered.  Some callers can do
// neither at call time: a host application that reserves all of its GPU
// memory up front and forbids allocation afterwards (game engines, plugin
// hosts with their own memory manager), or code that must not risk an
// allocation failing or stalling mid-frame.  dol_edt_mask_2d_noalloc gives
// them the same result with the scratch in a fixed device array that lives
// in the library image.
//
// The array holds kNoAllocMaxCells uint16 (16 MiB).  Every GPU that loads the
// library holds it until the process exits.  All calls on a device share it
// and it keeps the last call's contents; the x pass writes every cell it
// later reads, so nothing needs clearing.  Calls that overlap on the GPU
// (different streams, or different host threads on one device) race on the
// array: serialise them.
//
// The first call on a device does that device's set-up (the array's device
// address, the SM count, the column kernel's shared-memory limit); make that
// first call before capturing any stream into a CUDA graph.
#include <atomic>
#include <mutex>

#include "dol_b200.h"
#include "kernels.h"

namespace dolk {

constexpr size_t kNoAllocMaxCells = (size_t)8 << 20;   // 8,388,608 cells, e.g. 2896 x 2896 or 4096 x 2048
static __device__ __align__(256) uint16_t g_edt2_scratch[kNoAllocMaxCells];

// `ready` is stored (release) after scratch and sms are written; a caller
// that loads it true (acquire) sees both
struct NoAllocDevice {
    std::atomic<bool> ready{false};
    uint16_t* scratch = nullptr;   // device address of g_edt2_scratch on this device
    int sms = 0;
};
static NoAllocDevice g_noalloc[64];
static std::mutex g_noalloc_mu;

}  // namespace dolk

using namespace dolk;

extern "C" DOL_API dol_status dol_edt_mask_2d_noalloc(int w, int h, const uint32_t* mask, float* out, int form,
                                                      void* stream)
{
    if (w < 1 || h < 1) return (dol_status)set_error(DOL_ERR_INVALID_ARG, "dimensions must be >= 1 (got %d x %d)", w, h);
    if (w > 16384 || h > 16384)
        return (dol_status)set_error(DOL_ERR_UNSUPPORTED, "EDT dimensions are limited to 16384 (got %d x %d)", w, h);
    if ((size_t)w * h > kNoAllocMaxCells)
        return (dol_status)set_error(DOL_ERR_UNSUPPORTED,
                                     "image of %d x %d = %zu cells exceeds the no-allocation limit of %zu cells; "
                                     "use dol_edt_mask_2d with a workspace",
                                     w, h, (size_t)w * h, kNoAllocMaxCells);
    if (form != DOL_EDT_SQUARED && form != DOL_EDT_DIST && form != DOL_EDT_SIGNED)
        return (dol_status)set_error(DOL_ERR_INVALID_ARG, "form must be DOL_EDT_SQUARED, DOL_EDT_DIST or DOL_EDT_SIGNED");
    if (check_dev_ptr(mask, "mask") != DOL_OK) return DOL_ERR_INVALID_ARG;
    if (check_dev_ptr(out, "out") != DOL_OK) return DOL_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return (dol_status)set_error(DOL_ERR_CUDA, "no usable current device");
    }
    // set-up, once per device, with that device current: the array's name is
    // only a host-side stand-in; the kernels need its device address
    NoAllocDevice& nd = g_noalloc[dev];
    if (!nd.ready.load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!nd.ready.load(std::memory_order_relaxed)) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_edt2_scratch);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return (dol_status)set_error(DOL_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            }
            int sms = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return (dol_status)set_error(DOL_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
            }
            e = prepare_edt_mask_2d_plain();
            if (e != cudaSuccess) {
                cudaGetLastError();
                return (dol_status)set_error(DOL_ERR_CUDA, "cudaFuncSetAttribute (column kernel): %s",
                                             cudaGetErrorString(e));
            }
            nd.scratch = static_cast<uint16_t*>(p);
            nd.sms = sms;
            nd.ready.store(true, std::memory_order_release);
        }
    }
    cudaGetLastError();   // an earlier asynchronous error is not this call's
    launch_edt_mask_2d_plain(mask, out, w, h, form, nd.scratch, nd.sms, static_cast<cudaStream_t>(stream));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (dol_status)set_error(DOL_ERR_CUDA, "edt_mask_2d_noalloc: %s", cudaGetErrorString(e));
    return DOL_OK;
}
