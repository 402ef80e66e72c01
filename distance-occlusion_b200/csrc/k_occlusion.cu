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
// and (i, j, k-1), so any order that visits those three first gives the
// reference's values.  Two engines:
//   * the block wavefront (default): each plane is cut into blocks, the
//     blocks of one anti-diagonal run as one launch (k_occlusion_tiles2,
//     k_occlusion_blocks3), cells inside a block in a skewed wavefront;
//   * one CTA per plane (k_occlusion_sweep, k_occlusion_sweep1): thread t
//     owns C adjacent columns and walks the (slice, row) items in order,
//     skewed one step behind thread t-1, whose last column it takes from
//     shared memory (double-buffered by step parity); "up" stays in
//     registers and "back" is the thread's own output of h items before.
//     Rows of up to 1024 cells prefetch each item's loads a few steps ahead.
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

// One cell per thread along a row (the warp's stores to each plane are
// contiguous), rows handed out grid-stride; every plane gets the same values.
__global__ void k_init_dirw(const uint32_t* __restrict__ mask, float* __restrict__ dirw, int w, long long rows,
                            int planes, long long plane_stride)
{
    const int ws = words_per_row(w);
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const uint32_t* mrow = mask + r * ws;
        float* row = dirw + r * w;
        for (int x = threadIdx.x; x < w; x += blockDim.x) {
            const float v = (mrow[x >> 5] >> (x & 31)) & 1u ? 1.0f : 0.0f;
            for (int p = 0; p < planes; p++) row[p * plane_stride + x] = v;
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

// ---- block wavefront ------------------------------------------------------------------------
//
// The engines above keep one CTA per plane, so a sweep uses 4 or 8 SMs.  The
// block wavefront tiles each plane into blocks (in sweep order) and runs the
// blocks of one anti-diagonal per launch: a block's neighbours one step back
// in x, y or z lie on earlier diagonals, so when its launch starts every
// value it reads from outside itself is final, and no CTA ever waits for
// another.  Every cell still gets the reference's float operations on the
// same operand values, so the result is the same bit for bit whatever the
// order of the blocks.

// 2D: tiles of 32 x 32 cells, one warp each.  Lane r owns tile row r and at
// step s updates column s - r: its left neighbour is its own previous value,
// its upper neighbour lane r - 1's value of step s - 1 (a shuffle).  The tile
// is staged in shared memory with coalesced row loads and written back the
// same way; the row above and the column left of the tile come from earlier
// launches.  Launch `L` runs tiles (bx, by) with bx + by = L, bx = lo + blockIdx.x.
__global__ void __launch_bounds__(32) k_occlusion_tiles2(float* __restrict__ outp, int w, int h, int L, int lo)
{
    __shared__ float T[32][32];   // T[row][col]: lane r at step s touches bank (s - r) % 32
    const int bx = lo + blockIdx.x, by = L - bx;
    const int sweep = blockIdx.y;
    const int sx = sweep & 1, sy = (sweep >> 1) & 1;
    float* out = outp + (long long)sweep * w * h;
    const int r = threadIdx.x;
    const int i0 = bx * 32, j0 = by * 32;
    const int ni = min(32, w - i0), nj = min(32, h - j0);
    auto cell = [&](int i, int j) -> long long { return (long long)(sy ? h - 1 - j : j) * w + (sx ? w - 1 - i : i); };
    for (int rho = 0; rho < nj; rho++)
        if (r < ni) T[rho][r] = out[cell(i0 + r, j0 + rho)];
    const float upf = j0 > 0 && r < ni ? out[cell(i0 + r, j0 - 1)] : 0.0f;   // the row above, column r
    const float lf = i0 > 0 && r < nj ? out[cell(i0 - 1, j0 + r)] : 0.0f;    // the column to the left, row r
    __syncwarp();
    float v = 0.0f, prev = lf;
    const int S = ni + nj - 1;
    for (int s = 0; s < S; s++) {
        const float up_sh = __shfl_up_sync(0xFFFFFFFFu, v, 1);
        const float up_face = __shfl_sync(0xFFFFFFFFu, upf, s & 31);   // lane 0's column is s
        const int il = s - r;
        if (r < nj && il >= 0 && il < ni) {
            const float own = T[r][il];
            const float nv = i0 + il == 0 && j0 + r == 0 ? own   // the starting corner keeps its value
                                                         : occ_update(own, quad_combine(prev, r ? up_sh : up_face));
            T[r][il] = nv;
            prev = nv;
            v = nv;
        }
    }
    __syncwarp();
    for (int rho = 0; rho < nj; rho++)
        if (r < ni) out[cell(i0 + r, j0 + rho)] = T[rho][r];
}

// 3D: blocks of 32 x BY columns x bzs slices, one CTA of 32 x BY threads
// each (all 8 planes in one launch).  Thread (tx, ty) owns column (i, j) and
// at step s updates slice s - tx - ty of the block: "back" is its own
// previous value, "left" and "up" the values threads (tx-1, ty) and
// (tx, ty-1) published at step s - 1 (shared memory, double-buffered by step
// parity); on the block's faces they come from earlier launches.  Every
// global value a step needs is loaded kP steps ahead.  The grid spans two
// block axes (ax0, ax1: 0 = x, 1 = y, 2 = z); the third follows from L.
template <bool IO, int BY>
__global__ void __launch_bounds__(32 * BY, 1024 / (32 * BY))
    k_occlusion_blocks3(float* __restrict__ outp, const float* __restrict__ inp, int w, int h, int d, int bzs, int3 nb,
                        int ax0, int ax1, int L)
{
    constexpr int kP = 4;
    __shared__ float edge[2][BY][32];
    int b[3];
    b[0] = b[1] = b[2] = -1;
    b[ax0] = blockIdx.x;
    b[ax1] = blockIdx.y;
    const int ax2 = 3 - ax0 - ax1;
    b[ax2] = L - (int)blockIdx.x - (int)blockIdx.y;
    const int n2 = ax2 == 0 ? nb.x : (ax2 == 1 ? nb.y : nb.z);
    if (b[ax2] < 0 || b[ax2] >= n2) return;   // uniform: the whole CTA leaves
    const int sweep = blockIdx.z;
    const int sx = sweep & 1, sy = (sweep >> 1) & 1, sz = (sweep >> 2) & 1;
    const int dx = 1 - 2 * sx;
    const long long wh = (long long)w * h;
    const long long n = wh * d;
    float* out = outp + sweep * n;
    const float* in = IO ? inp + sweep * n : nullptr;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = b[0] * 32, j0 = b[1] * BY, k0 = b[2] * bzs;
    const int i = i0 + tx, j = j0 + ty;
    const int kn = min(bzs, d - k0);   // slices of the block
    const int S = kn + min(31, w - 1 - i0) + min(BY - 1, h - 1 - j0);   // the last column starts that late
    const bool has = i < w && j < h;
    const long long zs = sz ? -wh : wh;   // cell index step to the next slice in sweep order
    const long long ys = sy ? -(long long)w : (long long)w;
    const int z0 = sz ? d - 1 - k0 : k0;
    const long long c0 = has ? ((long long)z0 * h + (sy ? h - 1 - j : j)) * w + (sx ? w - 1 - i : i) : 0;
    const int lag = tx + ty;   // the thread updates slice s - lag at step s
    const bool lface = tx == 0 && i > 0, uface = ty == 0 && j > 0;
    const bool corner = i == 0 && j == 0 && k0 == 0;   // holds the plane's starting cell (slice 0)
    float own[kP], lf[kP], uf[kP], il[kP], iu[kP], ib[kP];
    float* pc = out + c0;   // the next cell to update
    const float* pf = pc;   // the next cell to fetch
    const float* qf = IO ? in + c0 : nullptr;
    int kf = 0;             // its slice in the block
    auto fetch = [&](int slot) {
        own[slot] = !IO || (corner && kf == 0) ? *pf : 0.0f;
        lf[slot] = lface ? pf[-dx] : 0.0f;
        uf[slot] = uface ? pf[-ys] : 0.0f;
        if (IO) {
            il[slot] = i ? qf[-dx] : 0.0f;
            iu[slot] = j ? qf[-ys] : 0.0f;
            ib[slot] = k0 + kf ? qf[-zs] : 0.0f;
            qf += zs;
        }
        pf += zs;
        kf++;
    };
#pragma unroll
    for (int u = 0; u < kP; u++)
        if (has && u - lag >= 0 && u - lag < kn) fetch(u);
    float prev = has && k0 > 0 ? pc[-zs] : 0.0f;   // "back" of the block's first slice
    bool first = corner;                            // the next cell is the plane's starting cell
    for (int s0 = 0; s0 < S; s0 += kP) {
#pragma unroll
        for (int u = 0; u < kP; u++) {
            const int s = s0 + u;
            if (s < S) {   // uniform
                const int q = s - lag;
                float v = 0.0f;
                if (has && q >= 0 && q < kn) {
                    const float left = tx ? edge[(s - 1) & 1][ty][tx - 1] : lf[u];
                    const float upv = ty ? edge[(s - 1) & 1][ty - 1][tx] : uf[u];
                    if (first) {
                        v = own[u];   // the starting corner keeps its value
                        first = false;
                    } else {
                        v = IO ? oct_combine_io(left, upv, prev, il[u], iu[u], ib[u])
                               : occ_update(own[u], oct_combine(left, upv, prev));
                        *pc = v;
                    }
                    prev = v;
                    pc += zs;
                }
                edge[s & 1][ty][tx] = v;
                if (has && s + kP - lag >= 0 && s + kP - lag < kn) fetch(u);
                __syncthreads();
            }
        }
    }
}

void launch_init_dirw(int dim, const uint32_t* mask, float* dirw, int w, int h, int d, cudaStream_t st)
{
    const long long rows = (long long)h * (dim == 3 ? d : 1);
    const int threads = w >= 256 ? 256 : (w + 31) / 32 * 32;
    const long long blocks = rows < (long long)g_num_sms * 32 ? rows : (long long)g_num_sms * 32;
    ProfScope ps("init_dirw", st);
    k_init_dirw<<<(int)blocks, threads, 0, st>>>(mask, dirw, w, rows, dim == 3 ? 8 : 4, (long long)w * rows);
}

// one CTA per plane (rows up to 4096 cells); the engine before the block wavefront
static void occ_planes(int dim, float* dirw, const float* in, int w, int h, int d, cudaStream_t st)
{
    const int C = w <= 1024 ? 1 : (w <= 2048 ? 2 : 4);
    int T = (w + C - 1) / C;
    T = (T + 31) & ~31;
    const int planes = dim == 3 ? 8 : 4;
    const int dd = dim == 3 ? d : 1;
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
        if (C == 2) DOL_OCC_CASE(2, false, 2);
        else DOL_OCC_CASE(2, false, 4);
    } else if (!in) {
        if (C == 2) DOL_OCC_CASE(3, false, 2);
        else DOL_OCC_CASE(3, false, 4);
    } else {
        if (C == 2) DOL_OCC_CASE(3, true, 2);
        else DOL_OCC_CASE(3, true, 4);
    }
#undef DOL_OCC_CASE
}

static void occ_tiles2(float* dirw, int w, int h, cudaStream_t st)
{
    const int nbx = (w + 31) / 32, nby = (h + 31) / 32;
    for (int L = 0; L < nbx + nby - 1; L++) {
        const int lo = max(0, L - (nby - 1)), hi = min(L, nbx - 1);
        k_occlusion_tiles2<<<dim3(hi - lo + 1, 4), 32, 0, st>>>(dirw, w, h, L, lo);
    }
}

template <bool IO, int BY>
static void occ_blocks3(float* dirw, const float* in, int w, int h, int d, int bzs, cudaStream_t st)
{
    const int3 nb = make_int3((w + 31) / 32, (h + BY - 1) / BY, (d + bzs - 1) / bzs);
    // the grid spans the two block axes with the fewest blocks; the third follows from the diagonal
    const int cnt[3] = {nb.x, nb.y, nb.z};
    int ax2 = 0;
    for (int a = 1; a < 3; a++)
        if (cnt[a] > cnt[ax2]) ax2 = a;
    const int ax0 = ax2 == 0 ? 1 : 0, ax1 = ax2 == 2 ? 1 : 2;
    const dim3 grid(cnt[ax0], cnt[ax1], 8), block(32, BY);
    for (int L = 0; L < nb.x + nb.y + nb.z - 2; L++)
        k_occlusion_blocks3<IO, BY><<<grid, block, 0, st>>>(dirw, in, w, h, d, bzs, nb, ax0, ax1, L);
}

void launch_occlusion_sweep(int dim, float* dirw, const float* in, int w, int h, int d, cudaStream_t st)
{
    ProfScope ps(in ? "occlusion_sweep_io" : "occlusion_sweep", st);
    const int t = tune_get(kTuneOcc, w);
    if (t == 1 && w <= kOccPlaneMaxWidth) {
        occ_planes(dim, dirw, in, w, h, d, st);
    } else if (dim == 2) {
        occ_tiles2(dirw, w, h, st);
    } else {
        // t > 1: slices per block (t % 1000); t >= 1000: blocks of 32 rows instead of 16
        const int bzs = t > 1 && t % 1000 ? min(t % 1000, 1024) : (d >= 256 ? 64 : kOccSlicesPerBlock);
        const bool rows32 = t >= 1000;
        if (in) {
            if (rows32) occ_blocks3<true, 32>(dirw, in, w, h, d, bzs, st);
            else occ_blocks3<true, 16>(dirw, in, w, h, d, bzs, st);
        } else {
            if (rows32) occ_blocks3<false, 32>(dirw, in, w, h, d, bzs, st);
            else occ_blocks3<false, 16>(dirw, in, w, h, d, bzs, st);
        }
    }
}

}  // namespace dolk
