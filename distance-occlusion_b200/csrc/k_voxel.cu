// k_voxel.cu -- triangle mesh to bitmask on the GPU.
//
// MSL::CreateBitMaskFromTriangles (MeshSupport.cpp:369-475): for every
// triangle, every cell of the w x h x d grid spanning bbox that lies in the
// triangle's cell range and whose box, grown by 0.000001 of a cell, meets the
// triangle gets its bit ORed into the mask; a triangle whose range is one
// cell sets that cell without a test, and one with an empty x range is
// skipped.  The overlap test (cTriCellIntersectDelta, :158-353) is the
// separating-axis test on the nine edge-by-axis cross products, split the
// reference's way into a per-slice part (z range), a per-row part (the x-axis
// crosses, y range) and a per-cell part (the y- and z-axis crosses, x range,
// then the triangle's plane).  Every float operation is the reference's, in
// its order, rounded on its own (__f*_rn: no contraction), so the bits are
// the reference's.
//
// One warp per triangle: all lanes prepare the triangle (the same values),
// walk its slices and rows together (the slice and row tests are uniform),
// and cover 32 consecutive x of a row at a time; the row's hits, gathered by
// a ballot, go to the mask as at most two atomicOr words.
#include "common.cuh"
#include "kernels.h"

namespace dolk {

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }   // MSL::Min
__device__ __forceinline__ float fmx(float a, float b) { return b < a ? a : b; }   // MSL::Max
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
// a*b - c*d and -(a*b) + c*d, each product rounded first
__device__ __forceinline__ float msub(float a, float b, float c, float d) { return sub(mul(a, b), mul(c, d)); }
__device__ __forceinline__ float nmadd(float a, float b, float c, float d) { return add(mul(-a, b), mul(c, d)); }

struct TriTest {
    V3 e[3], t[3], u[3], pmin, pmax, hw, n;
    float ndv_min, ndv_max, nd;
};

__device__ void tri_prepare(TriTest& s, V3 p1, V3 p2, V3 p3, V3 hw)
{
    s.hw = hw;
    s.e[0] = V3{sub(p2.x, p1.x), sub(p2.y, p1.y), sub(p2.z, p1.z)};
    s.e[1] = V3{sub(p3.x, p2.x), sub(p3.y, p2.y), sub(p3.z, p2.z)};
    s.e[2] = V3{sub(p1.x, p3.x), sub(p1.y, p3.y), sub(p1.z, p3.z)};
    // twice the area normal (:138-150): three products summed left to right
    s.n.x = add(add(mul(sub(p1.y, p2.y), add(p1.z, p2.z)), mul(sub(p2.y, p3.y), add(p2.z, p3.z))),
                mul(sub(p3.y, p1.y), add(p3.z, p1.z)));
    s.n.y = add(add(mul(sub(p1.z, p2.z), add(p1.x, p2.x)), mul(sub(p2.z, p3.z), add(p2.x, p3.x))),
                mul(sub(p3.z, p1.z), add(p3.x, p1.x)));
    s.n.z = add(add(mul(sub(p1.x, p2.x), add(p1.y, p2.y)), mul(sub(p2.x, p3.x), add(p2.y, p3.y))),
                mul(sub(p3.x, p1.x), add(p3.y, p1.y)));
    const V3 vmin{s.n.x > 0.0f ? -hw.x : hw.x, s.n.y > 0.0f ? -hw.y : hw.y, s.n.z > 0.0f ? -hw.z : hw.z};
    const V3 vmax{s.n.x > 0.0f ? hw.x : -hw.x, s.n.y > 0.0f ? hw.y : -hw.y, s.n.z > 0.0f ? hw.z : -hw.z};
    s.ndv_min = dot3(s.n, vmin);
    s.ndv_max = dot3(s.n, vmax);
    s.nd = dot3(s.n, p1);
    // edge k's three axis tests project two vertices each (:199-239): t from
    // (A[k][0], A[k][1], A[k][2]), u from (B[k][..]) for the x, y, z axes
    const V3 P[3] = {p1, p2, p3};
    const int A[3][3] = {{0, 0, 1}, {0, 0, 0}, {0, 0, 1}};
    const int B[3][3] = {{2, 2, 2}, {2, 2, 1}, {1, 1, 2}};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const V3 e = s.e[k];
        V3 t{msub(e.z, P[A[k][0]].y, e.y, P[A[k][0]].z), nmadd(e.z, P[A[k][1]].x, e.x, P[A[k][1]].z),
             msub(e.y, P[A[k][2]].x, e.x, P[A[k][2]].y)};
        V3 u{msub(e.z, P[B[k][0]].y, e.y, P[B[k][0]].z), nmadd(e.z, P[B[k][1]].x, e.x, P[B[k][1]].z),
             msub(e.y, P[B[k][2]].x, e.x, P[B[k][2]].y)};
        float q;
        if (t.x >= u.x) { q = t.x; t.x = u.x; u.x = q; }
        if (t.y >= u.y) { q = t.y; t.y = u.y; u.y = q; }
        if (t.z >= u.z) { q = t.z; t.z = u.z; u.z = q; }
        const V3 ae{fabsf(e.x), fabsf(e.y), fabsf(e.z)};
        const V3 r{add(mul(ae.z, hw.y), mul(ae.y, hw.z)), add(mul(ae.z, hw.x), mul(ae.x, hw.z)),
                   add(mul(ae.y, hw.x), mul(ae.x, hw.y))};
        s.t[k] = V3{sub(t.x, r.x), sub(t.y, r.y), sub(t.z, r.z)};
        s.u[k] = V3{add(u.x, r.x), add(u.y, r.y), add(u.z, r.z)};
    }
    s.pmin = V3{fmn(fmn(p1.x, p2.x), p3.x), fmn(fmn(p1.y, p2.y), p3.y), fmn(fmn(p1.z, p2.z), p3.z)};
    s.pmax = V3{fmx(fmx(p1.x, p2.x), p3.x), fmx(fmx(p1.y, p2.y), p3.y), fmx(fmx(p1.z, p2.z), p3.z)};
}

__device__ __forceinline__ bool hits_slice(const TriTest& s, float cz)
{
    return !(sub(s.pmin.z, cz) > s.hw.z || sub(s.pmax.z, cz) < -s.hw.z);
}

__device__ __forceinline__ bool hits_row(const TriTest& s, float cy, float cz)
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float dr = msub(s.e[k].z, cy, s.e[k].y, cz);
        if (s.t[k].x > dr || s.u[k].x < dr) return false;
    }
    return !(sub(s.pmin.y, cy) > s.hw.y || sub(s.pmax.y, cy) < -s.hw.y);
}

__device__ __forceinline__ bool hits_cell(const TriTest& s, V3 c)
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float dr = nmadd(s.e[k].z, c.x, s.e[k].x, c.z);
        if (s.t[k].y > dr || s.u[k].y < dr) return false;
        dr = msub(s.e[k].y, c.x, s.e[k].x, c.y);
        if (s.t[k].z > dr || s.u[k].z < dr) return false;
    }
    if (sub(s.pmin.x, c.x) > s.hw.x || sub(s.pmax.x, c.x) < -s.hw.x) return false;
    const float dd = sub(s.nd, dot3(s.n, c));
    return s.ndv_min <= dd && s.ndv_max >= dd;
}

struct VoxGrid {
    V3 cmin, cellw, inv, hw;
    int w, h, d, ws;
};

__global__ void __launch_bounds__(256) k_voxelize(const int* __restrict__ indices, const float* __restrict__ verts,
                                                  int tri_count, VoxGrid g, uint32_t* __restrict__ mask)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const size_t slice = (size_t)g.ws * g.h;
    for (long long t = warp; t < tri_count; t += nwarps) {
        V3 p[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const long long vi = indices ? (long long)indices[3 * t + k] : 3 * t + k;
            p[k] = V3{verts[3 * vi], verts[3 * vi + 1], verts[3 * vi + 2]};
        }
        const V3 bmin{fmn(fmn(p[0].x, p[1].x), p[2].x), fmn(fmn(p[0].y, p[1].y), p[2].y),
                      fmn(fmn(p[0].z, p[1].z), p[2].z)};
        const V3 bmax{fmx(fmx(p[0].x, p[1].x), p[2].x), fmx(fmx(p[0].y, p[1].y), p[2].y),
                      fmx(fmx(p[0].z, p[1].z), p[2].z)};
        const int x0 = max((int)floorf(mul(sub(bmin.x, g.cmin.x), g.inv.x)), 0);
        const int y0 = max((int)floorf(mul(sub(bmin.y, g.cmin.y), g.inv.y)), 0);
        const int z0 = max((int)floorf(mul(sub(bmin.z, g.cmin.z), g.inv.z)), 0);
        const int x1 = min((int)ceilf(mul(sub(bmax.x, g.cmin.x), g.inv.x)), g.w);
        const int y1 = min((int)ceilf(mul(sub(bmax.y, g.cmin.y), g.inv.y)), g.h);
        const int z1 = min((int)ceilf(mul(sub(bmax.z, g.cmin.z), g.inv.z)), g.d);
        if (x0 == x1) continue;
        if (x0 + 1 == x1 && y0 + 1 == y1 && z0 + 1 == z1) {   // a single cell: set without a test
            if (lane == 0) atomicOr(mask + slice * z0 + (size_t)g.ws * y0 + (x0 >> 5), 1u << (x0 & 31));
            continue;
        }
        TriTest s;
        tri_prepare(s, p[0], p[1], p[2], g.hw);
        for (int z = z0; z < z1; z++) {
            const float cz = add(g.cmin.z, mul(g.cellw.z, add((float)z, 0.5f)));
            if (!hits_slice(s, cz)) continue;
            for (int y = y0; y < y1; y++) {
                const float cy = add(g.cmin.y, mul(g.cellw.y, add((float)y, 0.5f)));
                if (!hits_row(s, cy, cz)) continue;
                uint32_t* row = mask + slice * z + (size_t)g.ws * y;
                for (int xb = x0; xb < x1; xb += 32) {
                    const int x = xb + lane;
                    bool hit = false;
                    if (x < x1) hit = hits_cell(s, V3{add(g.cmin.x, mul(g.cellw.x, add((float)x, 0.5f))), cy, cz});
                    const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit);
                    if (lane == 0 && b) {
                        const int sh = xb & 31;
                        atomicOr(row + (xb >> 5), b << sh);
                        if (sh && (b >> (32 - sh))) atomicOr(row + (xb >> 5) + 1, b >> (32 - sh));
                    }
                }
            }
        }
    }
}

void launch_voxelize(int tri_count, const int* indices, const float* verts, const float bbox[6], int w, int h, int d,
                     uint32_t* mask, cudaStream_t st)
{
    // the grid as the reference sets it up (:377-385), on the host in the same float operations
    VoxGrid g;
    g.cmin = V3{bbox[0], bbox[1], bbox[2]};
    const volatile float ex = bbox[3] - bbox[0], ey = bbox[4] - bbox[1], ez = bbox[5] - bbox[2];
    const volatile float fw = (float)w, fh = (float)h, fd = (float)d;
    g.cellw = V3{ex / fw, ey / fh, ez / fd};
    g.inv = V3{fw / ex, fh / ey, fd / ez};
    g.hw = V3{g.cellw.x * 0.500001f, g.cellw.y * 0.500001f, g.cellw.z * 0.500001f};
    g.w = w;
    g.h = h;
    g.d = d;
    g.ws = words_per_row(w);
    if (tri_count <= 0) return;
    long long blocks = ((long long)tri_count * 32 + 255) / 256;
    const long long cap = (long long)g_num_sms * 32;
    if (blocks > cap) blocks = cap;
    ProfScope ps("voxelize", st);
    k_voxelize<<<(int)blocks, 256, 0, st>>>(indices, verts, tri_count, g, mask);
}

}  // namespace dolk
