// k_occlusion.cu -- direction-weight initialisation and the occlusion sweeps.
//
// A direction-weight field has 4 (2D) or 8 (3D) planes of w*h[*d] floats;
// plane `sweep` holds the occlusion seen towards quadrant / octant `sweep`
// (bit 0: x decreasing, bit 1: y, bit 2: z).  InitDirWFromBitMask
// (DistanceOcclusionLib.cpp:1114-1146, :2507-2538) writes 1 on set cells and 0
// elsewhere in every plane.  OcclusionSweep (:1173-1209; 3D :2593-2650, the
// in/out form :2655-2737) walks a plane from its starting corner -- slices,
// rows, cells in sweep order -- and updates each cell from its already swept
// neighbours one step back along x ("left"), y ("up") and z ("back"),
// neighbours outside the field entering as 0, the corner cell left as it is:
//     in place:  x += (1 - x) * combine(left, up[, back])
//     in / out:  out = combine6(out neighbours, in neighbours)
// with the quadrant / octant combines of :1150-1169 and :2543-2567.
//
// Every cell depends on its left neighbour in the same row, so the result is
// bit-exact only with the reference's serial float chain along x: no
// reassociation, and every add / multiply rounded on its own (the __f*_rn
// intrinsics keep the compiler from contracting them into FMAs).  The
// parallelism is the wavefront: cell (i, j, k) needs (i-1, j, k), (i, j-1, k)
// and (i, j, k-1).  One CTA sweeps one plane (all planes at once); thread t
// owns C adjacent columns and walks the (slice, row) items in order, skewed
// one step behind thread t-1, whose last column it takes from shared memory
// (double-buffered by step parity); "up" stays in registers and "back" is
// the thread's own output of h items before.  Rows of up to 1024 cells (one
// column per thread) prefetch each item's loads a few steps ahead.
#include "common.cuh"
#include "kernels.h"

namespace dolk {

__device__ __forceinline__ float quad_combine(float a, float b)
{
    // 0.75f * ((a + b) - 1.0f * a * b)
    return __fmul_rn(0.75f, __fsub_rn(__fadd_rn(a, b), __fmul_rn(__fmul_rn(1.0f, a), b)));
}

__device__ __forceinline__ float oct_combine(float a, float b, float c)
{
    // 0.33333333f * (a + b + c - a * b * c)
    return __fmul_rn(0.33333333f, __fsub_rn(__fadd_rn(__fadd_rn(a, b), c), __fmul_rn(__fmul_rn(a, b), c)));
}

__device__ __forceinline__ float oct_combine_io(float oa, float ob, float oc, float ia, float ib, float ic)
{
    const float a = __fadd_rn(ia, __fmul_rn(__fsub_rn(1.0f, ia), oa));
    const float b = __fadd_rn(ib, __fmul_rn(__fsub_rn(1.0f, ib), ob));
    const float c = __fadd_rn(ic, __fmul_rn(__fsub_rn(1.0f, ic), oc));
    return __fmul_rn(0.3333333f, __fsub_rn(__fadd_rn(__fadd_rn(a, b), c), __fmul_rn(__fmul_rn(a, b), c)));
}

// x += (1 - x) * q
__device__ __forceinline__ float occ_update(float x, float q) { return __fadd_rn(x, __fmul_rn(__fsub_rn(1.0f, x), q)); }

// One word of mask (32 cells of a row) per thread; every plane gets the same values.
__global__ void k_init_dirw(const uint32_t* __restrict__ mask, float* __restrict__ dirw, int w, long long rows,
                            int planes, long long plane_stride)
{
    const int ws = words_per_row(w);
    const long long words = rows * ws;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < words;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / ws;
        const int k = (int)(i - r * ws);
        const uint32_t m = mask[i];
        const int x0 = 32 * k, n = min(32, w - x0);
        float* row = dirw + r * w + x0;
        for (int p = 0; p < planes; p++) {
            float* o = row + p * plane_stride;
            for (int b = 0; b < n; b++) o[b] = ((m >> b) & 1u) ? 1.0f : 0.0f;
        }
    }
}

template <int DIM, bool IO, int C>
__global__ void __launch_bounds__(1024) k_occlusion_sweep(float* __restrict__ outp, const float* __restrict__ inp, int w,
                                                          int h, int d)
{
    __shared__ float edge[2][1024];
    const int sweep = blockIdx.x;
    const int sx = sweep & 1, sy = (sweep >> 1) & 1, sz = (sweep >> 2) & 1;
    const int dx = 1 - 2 * sx, dy = 1 - 2 * sy, dz = 1 - 2 * sz;
    const long long wh = (long long)w * h;
    const long long n = wh * d;
    float* out = outp + sweep * n;
    const float* in = IO ? inp + sweep * n : nullptr;
    const int t = threadIdx.x;
    const int T = (w + C - 1) / C;   // threads holding columns (the rest only keep the barriers)
    const int ii0 = t * C;
    const int ncol = max(0, min(C, w - ii0));
    float up[C];
#pragma unroll
    for (int u = 0; u < C; u++) up[u] = 0.0f;
    const long long Q = (long long)d * h;
    int cj = 0, ck = 0;   // (row, slice) of the next item, kept as running counters
    for (long long s = 0; s < Q + T - 1; s++) {
        const long long q = s - t;
        float last = 0.0f;
        if (q >= 0 && q < Q && ncol > 0) {
            const int kk = ck, jj = cj;
            if (++cj == h) {
                cj = 0;
                ck++;
            }
            const int y = sy ? h - 1 - jj : jj, z = sz ? d - 1 - kk : kk;
            const long long rowbase = ((long long)z * h + y) * w;
            float left = ii0 > 0 ? edge[(s - 1) & 1][t - 1] : 0.0f;
#pragma unroll
            for (int u = 0; u < C; u++) {
                if (u < ncol) {
                    const int ii = ii0 + u;
                    const long long c = rowbase + (sx ? w - 1 - ii : ii);
                    const float upv = jj ? up[u] : 0.0f;
                    const float back = DIM == 3 && kk ? out[c - dz * wh] : 0.0f;
                    float v;
                    if (ii == 0 && jj == 0 && kk == 0) {
                        v = out[c];   // the starting corner keeps its value
                    } else if (IO) {
                        const float il = ii ? in[c - dx] : 0.0f;
                        const float iu = jj ? in[c - (long long)dy * w] : 0.0f;
                        const float ib = kk ? in[c - dz * wh] : 0.0f;
                        v = oct_combine_io(left, upv, back, il, iu, ib);
                        out[c] = v;
                    } else {
                        const float qv = DIM == 2 ? quad_combine(left, upv) : oct_combine(left, upv, back);
                        v = occ_update(out[c], qv);
                        out[c] = v;
                    }
                    up[u] = v;
                    left = v;
                }
            }
            last = left;
        }
        edge[s & 1][t] = last;
        __syncthreads();
    }
}

// The same sweep for rows of up to 1024 cells, one column per thread, with
// every global value an item needs loaded kP steps before its turn (the loop
// is unrolled by kP, so the ring of loads stays in registers): a step then
// waits on the barrier and the float chain, not on memory.  "back" (this
// thread's own output h items earlier) is prefetched only when h > kP, after
// it was written.
template <int DIM, bool IO>
__global__ void __launch_bounds__(1024) k_occlusion_sweep1(float* __restrict__ outp, const float* __restrict__ inp,
                                                           int w, int h, int d)
{
    constexpr int kP = 4;
    __shared__ float edge[2][1024];
    const int sweep = blockIdx.x;
    const int sx = sweep & 1, sy = (sweep >> 1) & 1, sz = (sweep >> 2) & 1;
    const int dx = 1 - 2 * sx, dy = 1 - 2 * sy, dz = 1 - 2 * sz;
    const long long wh = (long long)w * h;
    const long long n = wh * d;
    float* out = outp + sweep * n;
    const float* in = IO ? inp + sweep * n : nullptr;
    const int t = threadIdx.x;
    const bool has = t < w;
    const int x = sx ? w - 1 - t : t;
    const long long Q = (long long)d * h;
    const long long S = Q + w - 1;   // steps
    const bool pre_back = DIM == 3 && h > kP;
    float own[kP], bk[kP], il[kP], iu[kP], ib[kP];
    auto cell = [&](int jj, int kk) -> long long {
        const int y = sy ? h - 1 - jj : jj, z = sz ? d - 1 - kk : kk;
        return ((long long)z * h + y) * w + x;
    };
    auto fetch = [&](int jj, int kk, int slot) {
        const long long c = cell(jj, kk);
        own[slot] = out[c];
        if (pre_back) bk[slot] = kk ? out[c - dz * wh] : 0.0f;
        if (IO) {
            il[slot] = t ? in[c - dx] : 0.0f;
            iu[slot] = jj ? in[c - (long long)dy * w] : 0.0f;
            ib[slot] = kk ? in[c - dz * wh] : 0.0f;
        }
    };
    // items are (row jj, slice kk) in order; step s processes item s - t and
    // fetches item s - t + kP into the slot of step s % kP.  Both walk with
    // running counters (a 64-bit division per step cost more than the sweep).
    long long f = kP - t;   // the next item to fetch
    int fj = 0, fk = 0;
    if (f > 0) {
        fk = (int)(f / h);
        fj = (int)(f - (long long)fk * h);
    }
#pragma unroll
    for (int u = 0; u < kP; u++)   // items u - t: the first steps' slots
        if (has && u - t >= 0 && u - t < Q) fetch((u - t) % h, (u - t) / h, u);
    int cj = 0, ck = 0;   // the next item to process
    float up = 0.0f;
    for (long long s0 = 0; s0 < S; s0 += kP) {
#pragma unroll
        for (int u = 0; u < kP; u++) {
            const long long s = s0 + u;
            if (s < S) {   // uniform: every thread runs the same steps
                const long long q = s - t;
                float last = 0.0f;
                if (has && q >= 0 && q < Q) {
                    const int jj = cj, kk = ck;
                    const long long c = cell(jj, kk);
                    const float left = t ? edge[(s - 1) & 1][t - 1] : 0.0f;
                    const float upv = jj ? up : 0.0f;
                    float back = 0.0f;
                    if (DIM == 3 && kk) back = pre_back ? bk[u] : out[c - dz * wh];
                    float v;
                    if (t == 0 && jj == 0 && kk == 0) {
                        v = own[u];   // the starting corner keeps its value
                    } else if (IO) {
                        v = oct_combine_io(left, upv, back, il[u], iu[u], ib[u]);
                        out[c] = v;
                    } else {
                        const float qv = DIM == 2 ? quad_combine(left, upv) : oct_combine(left, upv, back);
                        v = occ_update(own[u], qv);
                        out[c] = v;
                    }
                    up = v;
                    last = v;
                    if (++cj == h) {
                        cj = 0;
                        ck++;
                    }
                }
                edge[s & 1][t] = last;
                if (has && f >= 0 && f < Q) {
                    fetch(fj, fk, u);
                    if (++fj == h) {
                        fj = 0;
                        fk++;
                    }
                }
                f++;
                __syncthreads();
            }
        }
    }
}

void launch_init_dirw(int dim, const uint32_t* mask, float* dirw, int w, int h, int d, cudaStream_t st)
{
    const long long rows = (long long)h * (dim == 3 ? d : 1);
    const long long words = rows * words_per_row(w);
    long long blocks = (words + 255) / 256;
    const long long cap = (long long)g_num_sms * 16;
    if (blocks > cap) blocks = cap;
    ProfScope ps("init_dirw", st);
    k_init_dirw<<<(int)blocks, 256, 0, st>>>(mask, dirw, w, rows, dim == 3 ? 8 : 4, (long long)w * rows);
}

void launch_occlusion_sweep(int dim, float* dirw, const float* in, int w, int h, int d, cudaStream_t st)
{
    const int C = w <= 1024 ? 1 : (w <= 2048 ? 2 : 4);
    int T = (w + C - 1) / C;
    T = (T + 31) & ~31;
    const int planes = dim == 3 ? 8 : 4;
    const int dd = dim == 3 ? d : 1;
    ProfScope ps(in ? "occlusion_sweep_io" : "occlusion_sweep", st);
    if (C == 1) {
        if (dim == 2)
            k_occlusion_sweep1<2, false><<<planes, T, 0, st>>>(dirw, in, w, h, 1);
        else if (!in)
            k_occlusion_sweep1<3, false><<<planes, T, 0, st>>>(dirw, in, w, h, dd);
        else
            k_occlusion_sweep1<3, true><<<planes, T, 0, st>>>(dirw, in, w, h, dd);
        return;
    }
#define DOL_OCC_CASE(DIMV, IOV, CV) \
    k_occlusion_sweep<DIMV, IOV, CV><<<planes, T, 0, st>>>(dirw, in, w, h, dd)
    if (dim == 2) {
        if (C == 1) DOL_OCC_CASE(2, false, 1);
        else if (C == 2) DOL_OCC_CASE(2, false, 2);
        else DOL_OCC_CASE(2, false, 4);
    } else if (!in) {
        if (C == 1) DOL_OCC_CASE(3, false, 1);
        else if (C == 2) DOL_OCC_CASE(3, false, 2);
        else DOL_OCC_CASE(3, false, 4);
    } else {
        if (C == 1) DOL_OCC_CASE(3, true, 1);
        else if (C == 2) DOL_OCC_CASE(3, true, 2);
        else DOL_OCC_CASE(3, true, 4);
    }
#undef DOL_OCC_CASE
}

}  // namespace dolk
