// tune.cu -- the launch-configuration table and the autotuner that fills it.
//
// Every kernel family here has launch parameters that change speed but never
// results (all kernels are exact for any of them): cells per thread for the
// row sweeps (and so threads per row), rows per CTA for the JumpFlood passes,
// threads per CTA for the EDT line passes, the CTA shape of the batched
// kernel.  The table maps (family, size bucket = ceil(log2 of the row or line
// length)) to a value per device; 0 means "not tuned", and launchers then use
// their built-in heuristic.  dol_autotune measures each candidate on a
// synthetic problem of the caller's shape (CUDA events, best of two runs) and
// keeps the fastest; dol_tune_set pins a value by hand.
#include <float.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "dol_b200.h"
#include "gen.cuh"
#include "kernels.h"

namespace dolk {

constexpr int kTuneDevices = 16;
constexpr int kTuneBuckets = 16;
static int g_tune[kTuneDevices][kTuneKinds][kTuneBuckets];
static std::mutex g_tune_mu;

static int bucket_of(int w)
{
    int b = 0;
    while (b < kTuneBuckets - 1 && (1 << b) < w) b++;
    return b;
}

static int cur_dev()
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return d >= 0 && d < kTuneDevices ? d : 0;
}

int tune_get(int kind, int w)
{
    if (kind < 0 || kind >= kTuneKinds) return 0;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return g_tune[cur_dev()][kind][bucket_of(w)];
}

void tune_put(int kind, int w, int value)
{
    if (kind < 0 || kind >= kTuneKinds) return;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[cur_dev()][kind][bucket_of(w)] = value;
}

// test hooks of the bounded waits (kernels.h); process-wide, read at launch
static WaitHooks g_wait_hooks = {-1, 1u << 22};

WaitHooks wait_hooks()
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return g_wait_hooks;
}

// candidate values per family
static std::vector<int> candidates(int kind, int w)
{
    switch (kind) {
        case kTuneDan2:
        case kTuneFs2:
        case kTuneDan3: {
            // CTA engine with 1/2/4/8 cells per thread, or (32) the single-warp engine
            std::vector<int> c;
            for (int s : {1, 2, 4, 8})
                if ((w + s - 1) / s <= 512) c.push_back(s);
            if (w <= (kind == kTuneDan3 ? 256 : 512)) c.push_back(32);
            return c;
        }
        case kTuneFs3: {   // the slice pipeline, then the anti-diagonal wavefront (negative)
            std::vector<int> c;
            for (int s : {1, 2, 4, 8})
                if ((w + s - 1) / s <= 256) c.push_back(s);
            for (int s : {1, 2, 4, 8})
                if ((w + s - 1) / s <= 256) c.push_back(-s);
            return c;
        }
        case kTuneJfa2: return {2, 4, 8, 16};
        case kTuneJfa3: return {2, 4, 8, 16, -2, -4, -8, -16};   // z walk, then one thread per cell
        case kTuneBatch: return {4, 8};
        case kTuneEdt: return {256, 512};
        case kTuneDanRows: return {4, 8, 16, 32, kDanSerial};
        case kTuneDanSlices: return {1, 4, 16, 64};
    }
    return {};
}

}  // namespace dolk

using namespace dolk;

// the batched kernel: a 256-image + 4-volume batch of the synthetic polygon /
// sphere generator, each CTA shape in turn
static dol_status tune_batch(cudaStream_t st)
{
    const int n2 = 256, n3 = 4, n = n2 + n3;
    std::vector<dol_batch_item> items(n);
    long long words = 0, dbytes = 0, cells = 0;
    dol_status s = dol_gen_batch(n2, n3, 13u, items.data(), &words, &dbytes, &cells, nullptr, st);
    if (s != DOL_OK) return s;
    void *dm = nullptr, *dd = nullptr, *df = nullptr, *ws = nullptr;
    const size_t wsb = dol_batch_workspace_size(n);
    if (cudaMalloc(&dm, words * 4) != cudaSuccess || cudaMalloc(&dd, dbytes) != cudaSuccess ||
        cudaMalloc(&df, cells * 4) != cudaSuccess || cudaMalloc(&ws, wsb) != cudaSuccess) {
        cudaGetLastError();
        for (void* p : {dm, dd, df, ws})
            if (p) cudaFree(p);
        return (dol_status)set_error(DOL_ERR_NO_MEMORY, "autotune scratch allocation failed");
    }
    s = dol_gen_batch(n2, n3, 13u, items.data(), nullptr, nullptr, nullptr, static_cast<uint32_t*>(dm), st);
    if (s == DOL_OK) s = dol_batch_prepare(n, items.data(), ws, wsb, st);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best_v = 4;
    float best_t = FLT_MAX;
    for (int v : candidates(kTuneBatch, 1024)) {
        if (s != DOL_OK) break;
        tune_put(kTuneBatch, 1024, v);
        s = dol_batch_run(n, static_cast<uint32_t*>(dm), dd, static_cast<float*>(df), ws, st);
        float t_best = FLT_MAX;
        for (int rep = 0; rep < 2 && s == DOL_OK; rep++) {
            cudaEventRecord(a, st);
            s = dol_batch_run(n, static_cast<uint32_t*>(dm), dd, static_cast<float*>(df), ws, st);
            cudaEventRecord(b, st);
            cudaEventSynchronize(b);
            float t = 0.0f;
            cudaEventElapsedTime(&t, a, b);
            if (t < t_best) t_best = t;
        }
        if (t_best < best_t) {
            best_t = t_best;
            best_v = v;
        }
    }
    tune_put(kTuneBatch, 1024, best_v);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamSynchronize(st);
    for (void* p : {dm, dd, df, ws})
        if (p) cudaFree(p);
    return s;
}

extern "C" {

DOL_API int dol_tune_get(int kind, int w) { return tune_get(kind, w); }

DOL_API void dol_test_wait_hooks(int stall_sweep, unsigned limit)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_wait_hooks.stall_sweep = stall_sweep >= 0 && stall_sweep < 8 ? stall_sweep : -1;
    g_wait_hooks.limit = limit ? limit : 1u << 22;
}

DOL_API void dol_tune_set(int kind, int w, int value) { tune_put(kind, w, value); }

DOL_API dol_status dol_autotune(int kind, int w, int h, int d, void* stream)
{
    if (kind < 0 || kind >= kTuneKinds) return (dol_status)set_error(DOL_ERR_INVALID_ARG, "unknown tuning family %d", kind);
    if (w < 1 || h < 1 || d < 1) return (dol_status)set_error(DOL_ERR_INVALID_ARG, "empty shape");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (kind == kTuneBatch) return tune_batch(st);
    const bool vol = kind == kTuneDan3 || kind == kTuneFs3 || kind == kTuneJfa3 || kind == kTuneEdt ||
                     ((kind == kTuneDanRows && d > 1) || kind == kTuneDanSlices);
    // a bounded synthetic problem of the caller's row / line shape
    int tw = w, th = h, td = vol ? d : 1;
    if (kind == kTuneFs2) th = h < 256 ? h : 256;
    if (kind == kTuneFs3) {
        // both engines are bound by their dependency chains (rows + slices
        // long) and the slice pipeline by its number of slices, so the ranking
        // changes with the shape (256 x 64 x 64 ranks 1 cell per thread first,
        // 256^3 2 cells): the caller's shape up to 2^25 cells, beyond that rows
        // and slices halved in turn
        while ((long long)tw * th * td > (1LL << 25) && (th > 64 || td > 64)) {
            if (th >= td)
                th = (th + 1) / 2;
            else
                td = (td + 1) / 2;
        }
    }
    if (kind == kTuneDan3) td = d < 32 ? d : 32;   // whole slices: the block schedule's row blocks
    if (kind == kTuneJfa2 && (long long)tw * th > (1LL << 22)) th = (int)((1LL << 22) / tw > 0 ? (1LL << 22) / tw : 1);
    if (kind == kTuneEdt) {
        // the EDT's line kernels are what the value picks, and their cost per
        // CTA depends on the y and z line lengths: narrow the volume along x
        // (independent column tiles) before shortening the lines
        while ((long long)tw * th * td > (1LL << 26) && tw > 64) tw = ((tw / 2 + 15) / 16) * 16;
    }
    if (kind == kTuneJfa3 || kind == kTuneEdt || kind == kTuneDanRows || kind == kTuneDanSlices) {
        while ((long long)tw * th * td > (1LL << 26) && td > 1) td = (td + 1) / 2;
    }
    const long long cells = (long long)tw * th * td;
    const size_t mwords = (size_t)((tw + 31) / 32) * th * td;

    // seeds: a sparse LCG scatter (delta methods), solids (FastSweep 3D) or
    // value noise (EDT)
    std::vector<uint32_t> hm(mwords, 0u);
    uint32_t seed = 77;
    const long long nseeds = cells / 64 + 1;
    for (long long i = 0; i < nseeds; i++) {
        seed = lcg_next(seed);
        int x = lcg_scale(seed, tw);
        seed = lcg_next(seed);
        int y = lcg_scale(seed, th);
        seed = lcg_next(seed);
        int z = lcg_scale(seed, td);
        hm[((size_t)z * th + y) * ((tw + 31) / 32) + (x >> 5)] |= 1u << (x & 31);
    }
    void *dm = nullptr, *dl = nullptr, *tmp = nullptr, *ws = nullptr;
    const size_t cell_bytes = vol ? 6 : 4;
    const bool dan = kind == kTuneDan2 || kind == kTuneDan3 || kind == kTuneDanRows || kind == kTuneDanSlices;
    size_t ws_bytes = kind == kTuneEdt ? edt_workspace_bytes(3, tw, th, td)
                      : dan            ? dan_blocks_workspace_bytes(vol ? 3 : 2, tw, th, td, 1)
                                       : fastsweep3_workspace_bytes(tw, th, td);
    bool ok = cudaMallocAsync(&dm, mwords * 4, st) == cudaSuccess &&
              cudaMallocAsync(&dl, (size_t)cells * (kind == kTuneEdt ? 4 : cell_bytes), st) == cudaSuccess &&
              cudaMallocAsync(&tmp, jumpflood_workspace_bytes(vol ? 3 : 2, tw, th, td), st) == cudaSuccess &&
              cudaMallocAsync(&ws, ws_bytes, st) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        for (void* p : {dm, dl, tmp, ws})
            if (p) cudaFreeAsync(p, st);
        return (dol_status)set_error(DOL_ERR_NO_MEMORY, "autotune scratch allocation failed");
    }
    if (kind == kTuneEdt) {
        dol_gen_value_noise_3d(tw, th, td, 16, 3u, static_cast<uint32_t*>(dm), st);
    } else if (kind == kTuneFs3) {
        // FastSweep 3D ranks its candidates differently on a scatter of single
        // seeds (1 cell per thread first) and on solids (2 cells on the 256^3
        // volume of boxes and spheres): tune it on solids, sized to the volume
        const int m = std::min(tw, std::min(th, td));
        dol_gen_shapes_3d(tw, th, td, 32, 32, std::max(1, 4 * m / 256), std::max(2, 40 * m / 256), 5u,
                          static_cast<uint32_t*>(dm), st);
    } else
        cudaMemcpyAsync(dm, hm.data(), mwords * 4, cudaMemcpyHostToDevice, st);
    int* err = nullptr;
    cudaMallocAsync((void**)&err, sizeof(int), st);

    auto run_once = [&]() {
        const int dim = vol ? 3 : 2;
        switch (kind) {
            case kTuneDan2:
            case kTuneDan3:   // through the entry path: block schedule or serial engine
                launch_init_border(dim, static_cast<uint32_t*>(dm), dl, tw, th, td, st);
                run_danielsson(dim, dl, tw, th, td, 2, ws, ws_bytes, err, st);
                break;
            case kTuneFs2:
                launch_init_border(2, static_cast<uint32_t*>(dm), dl, tw, th, 1, st);
                launch_fastsweep_2d(dl, tw, th, 2, st);
                break;
            case kTuneFs3:
                launch_init_border(3, static_cast<uint32_t*>(dm), dl, tw, th, td, st);
                launch_fastsweep_3d(dl, tw, th, td, 2, ws, err, st);
                break;
            case kTuneJfa2:
            case kTuneJfa3:
                launch_init_border(dim, static_cast<uint32_t*>(dm), dl, tw, th, td, st);
                launch_jumpflood(dim, dl, tmp, tw, th, td, 2, st);
                break;
            case kTuneEdt:
                launch_edt_mask(3, static_cast<uint32_t*>(dm), static_cast<float*>(dl), tw, th, td, DOL_EDT_SIGNED, ws,
                                err, st);
                break;
            case kTuneDanRows:
            case kTuneDanSlices:
                launch_init_border(dim, static_cast<uint32_t*>(dm), dl, tw, th, td, st);
                run_danielsson(dim, dl, tw, th, td, 2, ws, ws_bytes, err, st);
                break;
            case kTuneBatch:
                break;
        }
    };

    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best_v = 0;
    float best_t = FLT_MAX;
    const int saved = tune_get(kind, w);
    // a narrowed synthetic volume looks its value up under its own width:
    // give it each candidate too, and put its entry back afterwards
    const bool other_key = bucket_of(tw) != bucket_of(w);
    const int saved_tw = tune_get(kind, tw);
    for (int v : candidates(kind, w)) {
        tune_put(kind, w, v);
        if (other_key) tune_put(kind, tw, v);
        run_once();   // warm-up
        float t_best = FLT_MAX;
        for (int rep = 0; rep < 2; rep++) {
            cudaEventRecord(a, st);
            run_once();
            cudaEventRecord(b, st);
            cudaEventSynchronize(b);
            float t = 0.0f;
            cudaEventElapsedTime(&t, a, b);
            if (t < t_best) t_best = t;
        }
        if (t_best < best_t) {
            best_t = t_best;
            best_v = v;
        }
    }
    tune_put(kind, w, best_v ? best_v : saved);
    if (other_key) tune_put(kind, tw, saved_tw);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (void* p : {dm, dl, tmp, ws, (void*)err})
        if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (dol_status)set_error(DOL_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    return DOL_OK;
}

}  // extern "C"
