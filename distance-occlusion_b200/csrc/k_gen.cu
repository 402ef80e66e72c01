// k_gen.cu -- synthetic input volumes on the device (and the same bits on the
// host), plus the launch profiler used by the benchmark.
#include <float.h>

#include <mutex>
#include <string>
#include <vector>

#include "dol_b200.h"
#include "gen.cuh"
#include "kernels.h"

namespace dolk {

// One warp per 32 mask words; lane b evaluates cell 32k+b, a ballot forms the word.
template <class F>
__device__ void emit_mask_words(uint32_t* mask, int w, long long nwords, F bit_of)
{
    const int lane = threadIdx.x & 31;
    const int ws = words_per_row(w);
    long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < nwords; base += nwarps * 32) {
        uint32_t mine = 0;
        for (int q = 0; q < 32; q++) {
            long long wid = base + q;
            if (wid >= nwords) break;
            long long row = wid / ws;
            int x = 32 * (int)(wid - row * ws) + lane;
            bool b = x < w && bit_of(x, row);
            uint32_t word = __ballot_sync(0xFFFFFFFFu, b);
            if (lane == q) mine = word;
        }
        if (base + lane < nwords) mask[base + lane] = mine;
    }
}

__global__ void k_gen_noise(uint32_t* mask, NoiseSpec spec, long long nwords)
{
    emit_mask_words(mask, spec.w, nwords, [&](int x, long long row) {
        int z = (int)(row / spec.h), y = (int)(row - (long long)z * spec.h);
        return noise_bit(spec, x, y, z);
    });
}

__global__ void k_gen_shapes(uint32_t* mask, int w, int h, const Shape* shapes, int n, long long nwords)
{
    emit_mask_words(mask, w, nwords, [&](int x, long long row) {
        int z = (int)(row / h), y = (int)(row - (long long)z * h);
        return shape_bit(shapes, n, x, y, z);
    });
}

// ---------------------------------------------------------------- profiler ----
// When enabled, launchers bracket their kernels with events on the launch
// stream; dol_profile_end() waits for them and returns per-launch times.
struct ProfEntry {
    std::string name;
    cudaEvent_t a, b;
};
static std::mutex g_prof_mu;
static bool g_prof_on = false;
static std::vector<ProfEntry> g_prof;
static std::vector<cudaEvent_t> g_prof_pool;

static cudaEvent_t prof_event()
{
    if (!g_prof_pool.empty()) {
        cudaEvent_t e = g_prof_pool.back();
        g_prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

ProfScope::ProfScope(const char* name, cudaStream_t st) : st_(st)
{
    std::lock_guard<std::mutex> lock(g_prof_mu);
    if (!g_prof_on) return;
    ProfEntry e{name, prof_event(), prof_event()};
    cudaEventRecord(e.a, st);
    g_prof.push_back(e);
    idx_ = (int)g_prof.size() - 1;
}

ProfScope::~ProfScope()
{
    std::lock_guard<std::mutex> lock(g_prof_mu);
    if (idx_ < 0 || idx_ >= (int)g_prof.size()) return;
    cudaEventRecord(g_prof[idx_].b, st_);
}

}  // namespace dolk

using namespace dolk;

extern "C" {

DOL_API void dol_profile_begin(void)
{
    std::lock_guard<std::mutex> lock(g_prof_mu);
    for (auto& e : g_prof) {
        g_prof_pool.push_back(e.a);
        g_prof_pool.push_back(e.b);
    }
    g_prof.clear();
    g_prof_on = true;
}

DOL_API int dol_profile_end(char* names, size_t names_len, float* ms, int max_entries)
{
    std::lock_guard<std::mutex> lock(g_prof_mu);
    g_prof_on = false;
    int n = 0;
    size_t off = 0;
    for (auto& e : g_prof) {
        if (n >= max_entries) break;
        cudaEventSynchronize(e.b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e.a, e.b);
        ms[n] = t;
        if (names && off + e.name.size() + 1 < names_len) {
            memcpy(names + off, e.name.c_str(), e.name.size());
            off += e.name.size();
            names[off++] = '\n';
            names[off] = 0;
        }
        n++;
    }
    return n;
}

// ---- generators ---------------------------------------------------------------------------

// lattice values for the value-noise volume, drawn x fastest from the LCG
static std::vector<uint16_t> noise_lattice(int w, int h, int d, int L, uint32_t seed, int* gx, int* gy, int* gz)
{
    *gx = w / L + 2;
    *gy = h / L + 2;
    *gz = d / L + 2;
    std::vector<uint16_t> lat((size_t)(*gx) * (*gy) * (*gz));
    for (auto& v : lat) {
        seed = lcg_next(seed);
        v = (uint16_t)lcg_scale(seed, 65536);
    }
    return lat;
}

DOL_API dol_status dol_gen_value_noise_3d(int w, int h, int d, int spacing, uint32_t seed, uint32_t* mask, void* stream)
{
    if (w < 1 || h < 1 || d < 1 || spacing < 1 || spacing > 1024) return DOL_ERR_INVALID_ARG;
    int gx, gy, gz;
    std::vector<uint16_t> lat = noise_lattice(w, h, d, spacing, seed, &gx, &gy, &gz);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint16_t* dl = nullptr;
    if (cudaMallocAsync(&dl, lat.size() * 2, st) != cudaSuccess) return DOL_ERR_NO_MEMORY;
    cudaMemcpyAsync(dl, lat.data(), lat.size() * 2, cudaMemcpyHostToDevice, st);
    NoiseSpec spec{w, h, d, spacing, gx, gy, gz, dl};
    long long nwords = (long long)words_per_row(w) * h * d;
    long long blocks = (nwords + 255) / 256;
    if (blocks > 148LL * 32) blocks = 148LL * 32;
    k_gen_noise<<<(int)blocks, 256, 0, st>>>(mask, spec, nwords);
    cudaFreeAsync(dl, st);
    cudaStreamSynchronize(st);   // the lattice vector lives on this host stack frame
    return cudaGetLastError() == cudaSuccess ? DOL_OK : DOL_ERR_CUDA;
}

DOL_API void dol_gen_value_noise_3d_host(int w, int h, int d, int spacing, uint32_t seed, uint32_t* mask)
{
    int gx, gy, gz;
    std::vector<uint16_t> lat = noise_lattice(w, h, d, spacing, seed, &gx, &gy, &gz);
    NoiseSpec spec{w, h, d, spacing, gx, gy, gz, lat.data()};
    const int ws = words_per_row(w);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int k = 0; k < ws; k++) {
                uint32_t word = 0;
                for (int b = 0; b < 32 && 32 * k + b < w; b++)
                    if (noise_bit(spec, 32 * k + b, y, z)) word |= 1u << b;
                mask[((size_t)z * h + y) * ws + k] = word;
            }
}

// Boxes then spheres, sizes in [smin, smax], centres uniform, from the LCG in
// a fixed order: for each box cx, cy, cz, side x, side y, side z; for each
// sphere cx, cy, cz, radius.
static std::vector<Shape> shape_list(int w, int h, int d, int nbox, int nsph, int smin, int smax, uint32_t seed)
{
    std::vector<Shape> s;
    auto pick = [&](int limit) {
        seed = lcg_next(seed);
        return lcg_scale(seed, limit);
    };
    const int span = smax - smin + 1;
    for (int i = 0; i < nbox; i++) {
        Shape b{};
        b.kind = 0;
        b.cx = pick(w);
        b.cy = pick(h);
        b.cz = pick(d);
        b.a = smin + pick(span);
        b.b = smin + pick(span);
        b.c = smin + pick(span);
        s.push_back(b);
    }
    for (int i = 0; i < nsph; i++) {
        Shape b{};
        b.kind = 1;
        b.cx = pick(w);
        b.cy = pick(h);
        b.cz = pick(d);
        b.a = smin + pick(span);
        s.push_back(b);
    }
    return s;
}

DOL_API dol_status dol_gen_shapes_3d(int w, int h, int d, int nbox, int nsph, int smin, int smax, uint32_t seed,
                                     uint32_t* mask, void* stream)
{
    if (w < 1 || h < 1 || d < 1 || nbox < 0 || nsph < 0 || smin < 0 || smax < smin) return DOL_ERR_INVALID_ARG;
    std::vector<Shape> s = shape_list(w, h, d, nbox, nsph, smin, smax, seed);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Shape* ds = nullptr;
    size_t bytes = s.size() * sizeof(Shape);
    if (bytes && cudaMallocAsync(&ds, bytes, st) != cudaSuccess) return DOL_ERR_NO_MEMORY;
    if (bytes) cudaMemcpyAsync(ds, s.data(), bytes, cudaMemcpyHostToDevice, st);
    long long nwords = (long long)words_per_row(w) * h * d;
    long long blocks = (nwords + 255) / 256;
    if (blocks > 148LL * 32) blocks = 148LL * 32;
    k_gen_shapes<<<(int)blocks, 256, 0, st>>>(mask, w, h, ds, (int)s.size(), nwords);
    if (ds) cudaFreeAsync(ds, st);
    cudaStreamSynchronize(st);
    return cudaGetLastError() == cudaSuccess ? DOL_OK : DOL_ERR_CUDA;
}

DOL_API void dol_gen_shapes_3d_host(int w, int h, int d, int nbox, int nsph, int smin, int smax, uint32_t seed,
                                    uint32_t* mask)
{
    std::vector<Shape> s = shape_list(w, h, d, nbox, nsph, smin, smax, seed);
    const int ws = words_per_row(w);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int k = 0; k < ws; k++) {
                uint32_t word = 0;
                for (int b = 0; b < 32 && 32 * k + b < w; b++)
                    if (shape_bit(s.data(), (int)s.size(), 32 * k + b, y, z)) word |= 1u << b;
                mask[((size_t)z * h + y) * ws + k] = word;
            }
}

}  // extern "C"
