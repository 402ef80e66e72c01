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
    if (!g_prof_on || !name) return;   // an unnamed scope is not profiled
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

// ---- batch of uneven masks: star-shaped polygons and sphere volumes -----------------------

#include <algorithm>
#include <cmath>

namespace dolk {

// Item geometry for rasterisation.  Polygon vertices are fixed point (1/256
// cell) so the inside test is integer-exact on host and device.
struct GenShape {
    int kind;          // 0 polygon (2D), 1 spheres (3D)
    int nv;            // polygon vertices / spheres
    int first;         // index of the first vertex / sphere
    int pad;
};

// crossing-number test of the cell centre (x+1/2, y+1/2) against a polygon
DOL_HD bool polygon_bit(const int* vx, const int* vy, int nv, int x, int y)
{
    const long long px = 256LL * x + 128, py = 256LL * y + 128;
    bool in = false;
    for (int i = 0, j = nv - 1; i < nv; j = i++) {
        long long ax = vx[j], ay = vy[j], bx = vx[i], by = vy[i];
        if ((ay > py) != (by > py)) {
            // x of the edge at py is ax + (py-ay)(bx-ax)/(by-ay); compare without division
            long long lhs = (px - ax) * (by - ay), rhs = (py - ay) * (bx - ax);
            bool left = (by > ay) ? (lhs < rhs) : (lhs > rhs);
            if (left) in = !in;
        }
    }
    return in;
}

DOL_HD bool spheres_bit(const int* sp, int n, int x, int y, int z)
{
    for (int i = 0; i < n; i++) {
        long long dx = 2LL * x + 1 - 2LL * sp[4 * i], dy = 2LL * y + 1 - 2LL * sp[4 * i + 1],
                  dz = 2LL * z + 1 - 2LL * sp[4 * i + 2];
        long long r2 = 4LL * sp[4 * i + 3] * sp[4 * i + 3];
        if (dx * dx + dy * dy + dz * dz <= r2) return true;
    }
    return false;
}

__global__ void k_gen_batch(const dol_batch_item* items, const GenShape* shapes, const int* vx, const int* vy,
                            const int* spheres, uint32_t* masks)
{
    const dol_batch_item it = items[blockIdx.x];
    const GenShape g = shapes[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ws = words_per_row(it.w);
    const long long rows = (long long)it.h * it.d;
    uint32_t* m = masks + it.mask_word_offset;
    for (long long wid = warp; wid < rows * ws; wid += nw) {
        const long long row = wid / ws;
        const int k = (int)(wid - row * ws);
        const int x = 32 * k + lane;
        bool b = false;
        if (x < it.w) {
            if (g.kind == 0)
                b = polygon_bit(vx + g.first, vy + g.first, g.nv, x, (int)row);
            else
                b = spheres_bit(spheres + 4 * g.first, g.nv, x, (int)(row % it.h), (int)(row / it.h));
        }
        uint32_t word = __ballot_sync(0xFFFFFFFFu, b);
        if (lane == 0) m[wid] = word;
    }
}

struct BatchSpec {
    std::vector<dol_batch_item> items;
    std::vector<GenShape> shapes;
    std::vector<int> vx, vy, spheres;
    long long words = 0, delta_bytes = 0, cells = 0;
};

// The batch geometry from the reference's LCG: n2 images with side
// log-uniform in [32, 1024] and h = side * U[1, 2], each one star-shaped
// polygon with 3-12 vertices at sorted random angles and radii U[0.2, 0.45] *
// side about the centre; then n3 volumes with side uniform in [32, 128], each
// the union of 8 spheres (centres uniform, radii uniform in [side/8, side/3]).
static BatchSpec batch_spec(int n2, int n3, uint32_t seed)
{
    BatchSpec b;
    auto next = [&]() { seed = lcg_next(seed); return seed; };
    auto unit = [&]() { return (double)lcg_scale(next(), 1 << 24) / (double)(1 << 24); };
    auto pick = [&](int limit) { return lcg_scale(next(), limit); };
    auto add = [&](int w, int h, int d) {
        dol_batch_item it{};
        it.w = w; it.h = h; it.d = d;
        it.mask_word_offset = b.words;
        it.delta_byte_offset = b.delta_bytes;
        it.dist_offset = b.cells;
        long long cells = (long long)w * h * d;
        b.words += (long long)words_per_row(w) * h * d;
        b.delta_bytes += ((cells * (d > 1 ? 6 : 4)) + 15) / 16 * 16;
        b.cells += cells;
        b.items.push_back(it);
    };
    const double kTwoPi = 6.283185307179586;
    for (int i = 0; i < n2; i++) {
        int side = (int)std::floor(32.0 * std::pow(32.0, unit()));
        if (side > 1024) side = 1024;
        int h = (int)std::floor(side * (1.0 + unit()));
        add(side, h, 1);
        int nv = 3 + pick(10);
        std::vector<double> ang(nv);
        for (auto& a : ang) a = unit() * kTwoPi;
        std::sort(ang.begin(), ang.end());
        GenShape g{0, nv, (int)b.vx.size(), 0};
        const double cx = side * 0.5, cy = h * 0.5;
        for (int v = 0; v < nv; v++) {
            double r = (0.2 + 0.25 * unit()) * side;
            b.vx.push_back((int)std::lround(256.0 * (cx + r * std::cos(ang[v]))));
            b.vy.push_back((int)std::lround(256.0 * (cy + r * std::sin(ang[v]))));
        }
        b.shapes.push_back(g);
    }
    for (int i = 0; i < n3; i++) {
        int side = 32 + pick(97);
        add(side, side, side);
        GenShape g{1, 8, (int)(b.spheres.size() / 4), 0};
        for (int s = 0; s < 8; s++) {
            b.spheres.push_back(pick(side));
            b.spheres.push_back(pick(side));
            b.spheres.push_back(pick(side));
            b.spheres.push_back(side / 8 + pick(side / 3 - side / 8 + 1));
        }
        b.shapes.push_back(g);
    }
    return b;
}

}  // namespace dolk

extern "C" {

DOL_API dol_status dol_gen_batch(int n2, int n3, uint32_t seed, dol_batch_item* items, long long* total_mask_words,
                                 long long* total_delta_bytes, long long* total_cells, uint32_t* masks, void* stream)
{
    if (n2 < 0 || n3 < 0) return DOL_ERR_INVALID_ARG;
    BatchSpec b = batch_spec(n2, n3, seed);
    if (items) memcpy(items, b.items.data(), b.items.size() * sizeof(dol_batch_item));
    if (total_mask_words) *total_mask_words = b.words;
    if (total_delta_bytes) *total_delta_bytes = b.delta_bytes;
    if (total_cells) *total_cells = b.cells;
    if (!masks || b.items.empty()) return DOL_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto up = [&](const void* src, size_t bytes, void** dst) {
        if (bytes == 0) bytes = 4;
        if (cudaMallocAsync(dst, bytes, st) != cudaSuccess) return false;
        return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    };
    void *di = nullptr, *ds = nullptr, *dvx = nullptr, *dvy = nullptr, *dsp = nullptr;
    int zero[4] = {0, 0, 0, 0};
    bool ok = up(b.items.data(), b.items.size() * sizeof(dol_batch_item), &di) &&
              up(b.shapes.data(), b.shapes.size() * sizeof(GenShape), &ds) &&
              up(b.vx.empty() ? zero : b.vx.data(), b.vx.size() * 4, &dvx) &&
              up(b.vy.empty() ? zero : b.vy.data(), b.vy.size() * 4, &dvy) &&
              up(b.spheres.empty() ? zero : b.spheres.data(), b.spheres.size() * 4, &dsp);
    if (ok) {
        k_gen_batch<<<(int)b.items.size(), 256, 0, st>>>(static_cast<dol_batch_item*>(di), static_cast<GenShape*>(ds),
                                                         static_cast<int*>(dvx), static_cast<int*>(dvy),
                                                         static_cast<int*>(dsp), masks);
    }
    for (void* p : {di, ds, dvx, dvy, dsp})
        if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);   // the host copies of the geometry end with this call
    return ok && cudaGetLastError() == cudaSuccess ? DOL_OK : DOL_ERR_CUDA;
}

DOL_API void dol_gen_batch_host(int n2, int n3, uint32_t seed, uint32_t* masks)
{
    BatchSpec b = batch_spec(n2, n3, seed);
    for (size_t i = 0; i < b.items.size(); i++) {
        const dol_batch_item& it = b.items[i];
        const GenShape& g = b.shapes[i];
        const int ws = words_per_row(it.w);
        uint32_t* m = masks + it.mask_word_offset;
        for (long long row = 0; row < (long long)it.h * it.d; row++)
            for (int k = 0; k < ws; k++) {
                uint32_t word = 0;
                for (int bit = 0; bit < 32 && 32 * k + bit < it.w; bit++) {
                    int x = 32 * k + bit;
                    bool in = g.kind == 0 ? polygon_bit(b.vx.data() + g.first, b.vy.data() + g.first, g.nv, x, (int)row)
                                          : spheres_bit(b.spheres.data() + 4 * g.first, g.nv, x, (int)(row % it.h),
                                                        (int)(row / it.h));
                    if (in) word |= 1u << bit;
                }
                m[row * ws + k] = word;
            }
    }
}

}  // extern "C"
