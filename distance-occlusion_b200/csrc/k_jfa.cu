// k_jfa.cu -- JumpFlood passes and deltas -> distances.
//
// JumpFlood (DistanceOcclusionLib.cpp:782-908 for 2D, :2398-2472 for 3D) is a
// ping-pong stencil: every cell of a pass reads only the previous pass, so one
// thread per cell with the reference's fixed candidate order reproduces it
// exactly.  The driver keeps the reference's pass schedule: steps from
// FloorPow2(max dim - 1) halving to 1, plus one extra step-1 pass back into the
// caller's buffer when the last result sits in the ping-pong buffer.
#include "common.cuh"
#include "kernels.h"

namespace dolk {

__global__ void __launch_bounds__(512) k_jfa2(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int w,
                                              int h, int s, int cw)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (x >= w || y >= h) return;
    const int o = cw * s;
    auto at = [&](int xx, int yy) { return unpack2(__ldg(in + (long long)yy * w + xx)); };
    C2 best = at(x, y);
    int32_t bl = len(best);   // the incumbent's squared length, kept between candidates
    // closer(): a candidate wins only when strictly shorter
    auto consider = [&](C2 cand) {
        const int32_t cl = len(cand);
        if (bl > cl) {
            best = cand;
            bl = cl;
        }
    };
    // candidate order of :794-868
    if (x - s >= 0) {
        consider(add(at(x - s, y), -o, 0));
        if (y - s >= 0) consider(add(at(x - s, y - s), -o, -o));
        if (y + s < h) consider(add(at(x - s, y + s), -o, +o));
    }
    if (x + s < w) {
        consider(add(at(x + s, y), +o, 0));
        if (y - s >= 0) consider(add(at(x + s, y - s), +o, -o));
        if (y + s < h) consider(add(at(x + s, y + s), +o, +o));
    }
    if (y - s >= 0) consider(add(at(x, y - s), 0, -o));
    if (y + s < h) consider(add(at(x, y + s), 0, +o));
    out[(long long)y * w + x] = pack2(best);
}

__device__ __forceinline__ C3 load3(const int16_t* p, long long i)
{
    const int16_t* c = p + 3 * i;
    return C3{__ldg(c), __ldg(c + 1), __ldg(c + 2)};
}
__device__ __forceinline__ void store3(int16_t* p, long long i, C3 v)
{
    int16_t* c = p + 3 * i;
    c[0] = (int16_t)v.x;
    c[1] = (int16_t)v.y;
    c[2] = (int16_t)v.z;
}
// Between its first and last pass the 3D JumpFlood keeps cells in 8 bytes
// (x, y, z, unused): one aligned load per neighbour instead of three.
__device__ __forceinline__ C3 load3w(const uint2* p, long long i)
{
    const uint2 u = __ldg(p + i);
    return C3{(int)(int16_t)(u.x & 0xFFFFu), (int)(int16_t)(u.x >> 16), (int)(int16_t)(u.y & 0xFFFFu)};
}
__device__ __forceinline__ void store3w(uint2* p, long long i, C3 v)
{
    p[i] = make_uint2((uint32_t)(uint16_t)v.x | ((uint32_t)(uint16_t)v.y << 16), (uint32_t)(uint16_t)v.z);
}

// kWideIn / kWideOut: 8-byte cells (the ping-pong buffers) or the caller's 6-byte cells
template <bool kWideIn, bool kWideOut>
__global__ void __launch_bounds__(512) k_jfa3(const void* __restrict__ in, void* __restrict__ out, int w, int h, int d,
                                              int s, int cw)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int z = blockIdx.z;
    if (x >= w || y >= h) return;
    const long long plane = (long long)w * h;
    const long long idx = z * plane + (long long)y * w + x;
    auto ld = [&](long long i) -> C3 {
        return kWideIn ? load3w(static_cast<const uint2*>(in), i) : load3(static_cast<const int16_t*>(in), i);
    };
    C3 best = ld(idx);
    int32_t bl = len(best);   // the incumbent's squared length, kept between candidates
    // all offsets in {-s, 0, +s}^3 that stay inside, z outermost, x innermost,
    // skipping neighbours still at max (:2419-2438); a candidate wins only
    // when strictly shorter (closer())
    // (unrolled over the 27 offsets; an offset leaving the field is skipped)
    const bool zlo = z - s >= 0, zhi = z + s < d, ylo = y - s >= 0, yhi = y + s < h, xlo = x - s >= 0,
               xhi = x + s < w;
    const long long oz = (long long)s * plane, oy = (long long)s * w;
#pragma unroll
    for (int iz = -1; iz <= 1; iz++) {
        const bool vz = iz == 0 || (iz < 0 ? zlo : zhi);
#pragma unroll
        for (int iy = -1; iy <= 1; iy++) {
            const bool vy = iy == 0 || (iy < 0 ? ylo : yhi);
#pragma unroll
            for (int ix = -1; ix <= 1; ix++) {
                const bool vx = ix == 0 || (ix < 0 ? xlo : xhi);
                if (!(vz && vy && vx)) continue;
                const C3 c = ld(idx + iz * oz + iy * oy + ix * s);
                if (c.x == kMax3) continue;
                const C3 cand = add(c, cw * s * ix, cw * s * iy, cw * s * iz);
                const int32_t cl = len(cand);
                if (bl > cl) {
                    best = cand;
                    bl = cl;
                }
            }
        }
    }
    if (kWideOut)
        store3w(static_cast<uint2*>(out), idx, best);
    else
        store3(static_cast<int16_t*>(out), idx, best);
}

// The same pass walking z: a thread takes one column (x, y) and the cells
// z = r + i s of one residue class r (a chunk of kJfaChunk of them), and visits
// the slices r + j s in order, each slice's 9 neighbours of the column loaded
// once and applied to the three cells that read them -- as offset +s for cell
// j - 1, 0 for cell j and -s for cell j + 1.  A cell thus meets its candidates
// in the reference's order (its own value first, then the slice below, its
// own slice, the slice above, y then x within each), and the pass loads ~10
// values per cell instead of 27.
constexpr int kJfaChunk = 32;

template <bool kWideIn>
__device__ __forceinline__ C3 jfa_ld(const void* in, long long i)
{
    return kWideIn ? load3w(static_cast<const uint2*>(in), i) : load3(static_cast<const int16_t*>(in), i);
}

template <bool kWideIn, bool kWideOut>
__global__ void __launch_bounds__(512) k_jfa3z(const void* __restrict__ in, void* __restrict__ out, int w, int h, int d,
                                               int s, int cw, int nchunk)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (x >= w || y >= h) return;
    const int r = blockIdx.z / nchunk, chunk = blockIdx.z % nchunk;
    const int m = (d - r + s - 1) / s;   // cells r + i s < d
    const int i0 = chunk * kJfaChunk, i1 = min(m, i0 + kJfaChunk);
    if (i0 >= i1) return;
    const long long plane = (long long)w * h;
    const long long col = (long long)y * w + x;
    const bool ylo = y - s >= 0, yhi = y + s < h, xlo = x - s >= 0, xhi = x + s < w;
    const int o = cw * s;
    // the three cells a slice serves: A = j - 1 (offset +s), B = j (0), C = j + 1 (-s)
    C3 bA{0, 0, 0}, bB{0, 0, 0}, bC{0, 0, 0};
    int32_t lA = 0, lB = 0, lC = 0;
    auto consider = [](C3& best, int32_t& bl, const C3& cand) {
        const int32_t cl = len(cand);
        if (bl > cl) {   // strictly shorter (closer())
            best = cand;
            bl = cl;
        }
    };
    for (int j = i0 - 1; j <= i1; j++) {
        const bool hasA = j - 1 >= i0, hasB = j >= i0 && j < i1, hasC = j + 1 < i1;
        if (hasC) {   // cell j + 1 starts from its own value
            bC = jfa_ld<kWideIn>(in, (long long)(r + (j + 1) * s) * plane + col);
            lC = len(bC);
        }
        if (j >= 0 && j < m) {   // slice r + j s exists: its 9 neighbours of the column
            const long long base = (long long)(r + j * s) * plane + col;
#pragma unroll
            for (int iy = -1; iy <= 1; iy++) {
                const bool vy = iy == 0 || (iy < 0 ? ylo : yhi);
#pragma unroll
                for (int ix = -1; ix <= 1; ix++) {
                    const bool vx = ix == 0 || (ix < 0 ? xlo : xhi);
                    if (!(vy && vx)) continue;
                    const C3 c = jfa_ld<kWideIn>(in, base + (long long)iy * s * w + ix * s);
                    if (c.x == kMax3) continue;
                    const int cx = trunc16(c.x + o * ix), cy = trunc16(c.y + o * iy);
                    if (hasC) consider(bC, lC, C3{cx, cy, trunc16(c.z - o)});
                    if (hasB) consider(bB, lB, C3{cx, cy, c.z});
                    if (hasA) consider(bA, lA, C3{cx, cy, trunc16(c.z + o)});
                }
            }
        }
        if (hasA) {   // cell j - 1 has seen its three slices
            const long long idx = (long long)(r + (j - 1) * s) * plane + col;
            if (kWideOut)
                store3w(static_cast<uint2*>(out), idx, bA);
            else
                store3(static_cast<int16_t*>(out), idx, bA);
        }
        bA = bB;
        lA = lB;
        bB = bC;
        lB = lC;
    }
}

size_t jumpflood_workspace_bytes(int dim, int w, int h, int d)
{
    const size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    if (dim == 2) return cells * sizeof(uint32_t);
    return 2 * (((cells * sizeof(uint2)) + 255) & ~(size_t)255);
}

static int floor_pow2(int v)
{
    v |= v >> 1;
    v |= v >> 2;
    v |= v >> 4;
    v |= v >> 8;
    v |= v >> 16;
    return (v + 1) >> 1;
}

void launch_jumpflood(int dim, void* deltas, void* temp, int w, int h, int d, int cw, cudaStream_t st)
{
    int m = w > h ? w : h;
    if (dim == 3 && d > m) m = d;
    // rows per CTA (32 x ry threads): tuned, else 8
    int ry = tune_get(dim == 2 ? kTuneJfa2 : kTuneJfa3, w);
    const bool per_cell = dim == 3 && ry < 0;   // 3D, negative tuned values: one thread per cell (k_jfa3)
    if (per_cell) ry = -ry;
    if (ry != 2 && ry != 4 && ry != 8 && ry != 16) ry = 8;
    // the reference's schedule: steps FloorPow2(m - 1) .. 1 ping-ponging with
    // the caller's buffer, plus one step-1 pass when the result would end in temp
    int steps[40], np = 0;
    for (int s = floor_pow2(m - 1); s > 0; s /= 2) steps[np++] = s;
    if (np & 1) steps[np++] = 1;
    if (dim == 2) {
        void* a = deltas;
        void* b = temp;
        const dim3 grid((w + 31) / 32, (h + ry - 1) / ry);
        for (int i = 0; i < np; i++) {
            ProfScope ps("jumpflood_pass", st);
            k_jfa2<<<grid, 32 * ry, 0, st>>>(static_cast<const uint32_t*>(a), static_cast<uint32_t*>(b), w, h, steps[i],
                                             cw);
            void* t = a;
            a = b;
            b = t;
        }
        return;
    }
    // 3D: the caller's 6-byte cells -> 8-byte ping-pong buffers -> the caller's cells
    const size_t cells = (size_t)w * h * d;
    uint2* wb[2] = {static_cast<uint2*>(temp),
                    reinterpret_cast<uint2*>(static_cast<char*>(temp) + (((cells * sizeof(uint2)) + 255) & ~(size_t)255))};
    const dim3 grid((w + 31) / 32, (h + ry - 1) / ry, d);
    for (int i = 0; i < np; i++) {
        ProfScope ps("jumpflood_pass", st);
        const bool first = i == 0, last = i == np - 1;
        const void* src = first ? deltas : wb[(i - 1) & 1];
        void* dst = last ? deltas : wb[i & 1];
        const int sv = steps[i];
        if (per_cell) {
            if (first)
                k_jfa3<false, true><<<grid, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw);
            else if (last)
                k_jfa3<true, false><<<grid, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw);
            else
                k_jfa3<true, true><<<grid, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw);
            continue;
        }
        // z walk: residue classes of z mod s, chunks of kJfaChunk cells along each
        const int nres = sv < d ? sv : d;
        const int nchunk = ((d + sv - 1) / sv + kJfaChunk - 1) / kJfaChunk;
        const dim3 gz((w + 31) / 32, (h + ry - 1) / ry, (unsigned)(nres * nchunk));
        if (first)
            k_jfa3z<false, true><<<gz, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw, nchunk);
        else if (last)
            k_jfa3z<true, false><<<gz, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw, nchunk);
        else
            k_jfa3z<true, true><<<gz, 32 * ry, 0, st>>>(src, dst, w, h, d, sv, cw, nchunk);
    }
}

// ---- deltas -> distances (DistanceOcclusionTool.cpp:46-61, sign :1262/:1392) ----

template <int kDim>
__global__ void __launch_bounds__(256) k_deltas_to_dist(const void* __restrict__ deltas, int cw,
                                                        const uint32_t* __restrict__ sign_mask, float* __restrict__ out,
                                                        int w, long long rows)
{
    const int ws = words_per_row(w);
    const long long n = rows * w;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int32_t l;
        if (kDim == 2) {
            l = len(unpack2(__ldg(static_cast<const uint32_t*>(deltas) + i)));
        } else {
            l = len(load3(static_cast<const int16_t*>(deltas), i));
        }
        float r = sqrtf((float)l);
        if (cw != 1) r = __fdiv_rn(r, (float)cw);
        if (sign_mask) {
            long long row = i / w;
            int x = (int)(i - row * w);
            if ((__ldg(sign_mask + row * ws + (x >> 5)) >> (x & 31)) & 1u) r = -r;
        }
        out[i] = r;
    }
}

void launch_deltas_to_dist(int dim, const void* deltas, int cw, const uint32_t* sign_mask, float* out, int w, int h,
                           int d, cudaStream_t st)
{
    long long rows = (long long)h * (dim == 3 ? d : 1);
    long long n = rows * w;
    long long blocks = (n + 255) / 256;
    long long cap = (long long)g_num_sms * 32;
    int grid = (int)(blocks < cap ? blocks : cap);
    ProfScope ps("deltas_to_dist", st);
    if (dim == 2)
        k_deltas_to_dist<2><<<grid, 256, 0, st>>>(deltas, cw, sign_mask, out, w, rows);
    else
        k_deltas_to_dist<3><<<grid, 256, 0, st>>>(deltas, cw, sign_mask, out, w, rows);
}

// ---- two-pass signed distance: Dist(exterior) - Dist(interior) ----
// The tool's -S path (GenerateSignedDistance, DistanceOcclusionTool.cpp:1082-1123
// 2D, :1197-1232 3D; Dist :54-61): deltas to set cells and deltas to clear cells,
// each with cw = 1, give sqrtf of each squared length, subtracted in float.
template <int kDim>
__global__ void __launch_bounds__(256) k_two_pass_dist(const void* __restrict__ ext, const void* __restrict__ intr,
                                                       float* __restrict__ out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int32_t a, b;
        if (kDim == 2) {
            a = len(unpack2(__ldg(static_cast<const uint32_t*>(ext) + i)));
            b = len(unpack2(__ldg(static_cast<const uint32_t*>(intr) + i)));
        } else {
            a = len(load3(static_cast<const int16_t*>(ext), i));
            b = len(load3(static_cast<const int16_t*>(intr), i));
        }
        out[i] = __fsub_rn(sqrtf((float)a), sqrtf((float)b));
    }
}

void launch_two_pass_dist(int dim, const void* ext, const void* intr, float* out, long long cells, cudaStream_t st)
{
    long long blocks = (cells + 255) / 256;
    long long cap = (long long)g_num_sms * 32;
    int grid = (int)(blocks < cap ? blocks : cap);
    ProfScope ps("two_pass_dist", st);
    if (dim == 2)
        k_two_pass_dist<2><<<grid, 256, 0, st>>>(ext, intr, out, cells);
    else
        k_two_pass_dist<3><<<grid, 256, 0, st>>>(ext, intr, out, cells);
}

}  // namespace dolk
