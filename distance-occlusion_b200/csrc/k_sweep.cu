// k_sweep.cu -- Danielsson and FastSweep, exact.
//
// Danielsson (DistanceOcclusionLib.cpp:702-778 2D, :2264-2394 3D) and FastSweep
// 2D (:633-697) are serial in the sweep axis: every row needs the whole
// previous row.  One CTA walks the rows of an image (or the slices and rows of
// a volume); each thread keeps S consecutive cells of the current and previous
// row in registers, so the vertical (and z) pulls are thread-local and only the
// x passes talk across threads (row_pass in scan.cuh, exact).  The next row is
// loaded while the current one is scanned.
//
// FastSweep 3D (:2186-2260) has more parallelism: row (y, z) of an octant
// sweep needs only row (y-1, z) and row (y, z-1) of the same sweep, so rows on
// an anti-diagonal y+z = c are independent.  k_fastsweep3 runs one octant per
// launch with persistent CTAs that claim rows in anti-diagonal order from an
// atomic counter and wait (bounded) on per-row ready flags.  A row is only
// claimed by a running CTA and every row it waits on was claimed earlier, so
// the earliest unfinished row can always proceed.
#include <limits.h>

#include "kernels.h"
#include "scan.cuh"

namespace dolk {

// ---------------------------------------------------------------- helpers ----

template <class Cell, int S, class P>
__device__ __forceinline__ void load_row(Cell (&dst)[S], const P* base, long long row_first, int n)
{
#pragma unroll
    for (int s = 0; s < S; s++)
        if (s < n) dst[s] = cell_load(base, row_first + s);
}
template <class Cell, int S, class P>
__device__ __forceinline__ void store_row(P* base, long long row_first, const Cell (&src)[S], int n)
{
#pragma unroll
    for (int s = 0; s < S; s++)
        if (s < n) cell_store(base, row_first + s, src[s]);
}
// L2-coherent loads for rows written by other CTAs of the same launch
__device__ __forceinline__ C3 cell_load_cg(const int16_t* p, long long i)
{
    const int16_t* c = p + 3 * i;
    return C3{__ldcg(c), __ldcg(c + 1), __ldcg(c + 2)};
}

// ------------------------------------------------------------ Danielsson 2D ----
// Rows 1..h-1 going down, then h-2..0 going up (:709-777): one "step" per row,
// the row taking the previous step's row with a y offset of -cw (down) or
// +cw (up), then an x pass to the right and one to the left.  The next step's
// row is loaded during the current one, and each pass posts what the next
// pass needs (row_pass), so a step costs two barriers when the passes settle
// in one round.

// One CTA runs the whole 2D Danielsson of one image (used by the single-image
// kernel and by the batched kernel).
template <int S>
__device__ __forceinline__ void danielsson2_cta(uint32_t* __restrict__ dl, int w, int h, int cw, ScanShared<C2>& sh)
{
    const int t = threadIdx.x;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    if (h < 2) return;
    const int steps = 2 * (h - 1);
    auto row_of = [&](int i) { return i < h - 1 ? i + 1 : 2 * h - 3 - i; };
    auto dy_of = [&](int i) { return i < h - 1 ? -cw : cw; };
    C2 P[S], C[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = V[s] = R[s] = D[s] = C2{0, 0};

    load_row<C2, S>(P, dl, x0, n);
    load_row<C2, S>(C, dl, (long long)row_of(0) * w + x0, n);
#pragma unroll
    for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, dy_of(0)));
    int g = 0;
    if (active) sh.guess[g][t] = seg_edge<C2, S, +1>(V, n);
    __syncthreads();
    for (int i = 0; i < steps; i++) {
        const int y = row_of(i);
        const bool more = i + 1 < steps;
        const int dyn = more ? dy_of(i + 1) : 0;
        if (more) load_row<C2, S>(C, dl, (long long)row_of(i + 1) * w + x0, n);
        const C2 in0 = (active && t > 0) ? sh.guess[g][t - 1] : V[0];
        row_pass<C2, S, false, +1>(R, V, t, nseg, n, cw, sh, D, in0, [&](const C2 (&X)[S]) {
            if (active) sh.guess[g ^ 1][t] = X[0];
        });
        g ^= 1;
        const C2 in1 = (active && t + 1 < nseg) ? sh.guess[g][t + 1] : R[0];
        row_pass<C2, S, false, -1>(P, R, t, nseg, n, cw, sh, D, in1, [&](const C2 (&X)[S]) {
            if (more && active)
                sh.guess[g ^ 1][t] = closer(seg_edge<C2, S, +1>(C, n), add(seg_edge<C2, S, +1>(X, n), 0, dyn));
        });
        g ^= 1;
        store_row<C2, S>(dl, (long long)y * w + x0, P, n);
        if (more) {
#pragma unroll
            for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, dyn));
        }
    }
}

template <int S>
__global__ void __launch_bounds__(512) k_danielsson2(uint32_t* __restrict__ dl, int w, int h, int cw)
{
    __shared__ ScanShared<C2> sh;
    danielsson2_cta<S>(dl, w, h, cw, sh);
}

// ------------------------------------------------------------ Danielsson 3D ----
// Slices 1..d-1 then d-2..0 (:2355-2393); each slice takes the neighbouring
// slice's cell with the z offset, then runs the 2D steps over its rows
// (:2264-2345).  The z pull is folded into the first load of each row (rows of
// the down sweep); the up sweep reads the down sweep's results.

template <int S>
__device__ __forceinline__ void danielsson3_cta(int16_t* __restrict__ dl, int w, int h, int d, int cw,
                                                ScanShared<C3>& sh)
{
    const int t = threadIdx.x;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    const long long plane = (long long)w * h;
    const int steps = 2 * (h - 1);
    auto row_of = [&](int i) { return i < h - 1 ? i + 1 : 2 * h - 3 - i; };
    auto dy_of = [&](int i) { return i < h - 1 ? -cw : cw; };
    C3 P[S], C[S], Q[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = Q[s] = V[s] = R[s] = D[s] = C3{0, 0, 0};

    for (int pass = 0; pass < 2; pass++) {
        const int dz = pass == 0 ? -cw : +cw;
        for (int k = 1; k < d; k++) {
            const int z = pass == 0 ? k : d - 1 - k;
            const int zp = pass == 0 ? z - 1 : z + 1;
            const long long sb = z * plane, pb = (long long)zp * plane;
            // row 0: z pull only
            load_row<C3, S>(C, dl, sb + x0, n);
            load_row<C3, S>(Q, dl, pb + x0, n);
#pragma unroll
            for (int s = 0; s < S; s++) P[s] = closer(C[s], add(Q[s], 0, 0, dz));
            store_row<C3, S>(dl, sb + x0, P, n);
            if (h < 2) continue;
            // first step: row 1 of the down sweep (z pull, then y pull)
            load_row<C3, S>(C, dl, sb + (long long)w + x0, n);
            load_row<C3, S>(Q, dl, pb + (long long)w + x0, n);
#pragma unroll
            for (int s = 0; s < S; s++) V[s] = closer(closer(C[s], add(Q[s], 0, 0, dz)), add(P[s], 0, -cw, 0));
            int g = 0;
            __syncthreads();   // the previous slice's last pass may still read the guess slots
            if (active) sh.guess[g][t] = seg_edge<C3, S, +1>(V, n);
            __syncthreads();
            for (int i = 0; i < steps; i++) {
                const int y = row_of(i);
                const bool more = i + 1 < steps;
                const bool next_down = more && i + 1 < h - 1;
                const int dyn = more ? dy_of(i + 1) : 0;
                if (more) {
                    const long long off = (long long)row_of(i + 1) * w + x0;
                    load_row<C3, S>(C, dl, sb + off, n);
                    if (next_down) load_row<C3, S>(Q, dl, pb + off, n);
                }
                const C3 in0 = (active && t > 0) ? sh.guess[g][t - 1] : V[0];
                row_pass<C3, S, false, +1>(R, V, t, nseg, n, cw, sh, D, in0, [&](const C3 (&X)[S]) {
                    if (active) sh.guess[g ^ 1][t] = X[0];
                });
                g ^= 1;
                const C3 in1 = (active && t + 1 < nseg) ? sh.guess[g][t + 1] : R[0];
                row_pass<C3, S, false, -1>(P, R, t, nseg, n, cw, sh, D, in1, [&](const C3 (&X)[S]) {
                    if (more && active) {
                        C3 c = seg_edge<C3, S, +1>(C, n);
                        if (next_down) c = closer(c, add(seg_edge<C3, S, +1>(Q, n), 0, 0, dz));
                        sh.guess[g ^ 1][t] = closer(c, add(seg_edge<C3, S, +1>(X, n), 0, dyn, 0));
                    }
                });
                g ^= 1;
                store_row<C3, S>(dl, sb + (long long)y * w + x0, P, n);
                if (more) {
#pragma unroll
                    for (int s = 0; s < S; s++) {
                        C3 c = next_down ? closer(C[s], add(Q[s], 0, 0, dz)) : C[s];
                        V[s] = closer(c, add(P[s], 0, dyn, 0));
                    }
                }
            }
        }
    }
}

template <int S>
__global__ void __launch_bounds__(512) k_danielsson3(int16_t* __restrict__ dl, int w, int h, int d, int cw)
{
    __shared__ ScanShared<C3> sh;
    danielsson3_cta<S>(dl, w, h, d, cw, sh);
}

// ------------------------------------------------------------- FastSweep 2D ----
// Four quadrant sweeps; the first row of each sweep is left as is; each later
// row takes the previous row's cell, then along x the previous cell of the row
// and the diagonal cell of the previous row, in that order (:655-693).  The
// diagonal candidate of a segment's first cell is its predecessor's boundary
// cell of the previous row, posted during the previous row's pass.

template <int S>
__global__ void __launch_bounds__(512) k_fastsweep2(uint32_t* __restrict__ dl, int w, int h, int cw)
{
    __shared__ ScanShared<C2> sh;
    const int t = threadIdx.x;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    C2 P[S], C[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = V[s] = R[s] = D[s] = C2{0, 0};
    if (h < 2) return;

    for (int sweep = 0; sweep < 4; sweep++) {
        const int dx = (sweep & 1) ? -1 : 1, dy = (sweep & 2) ? -1 : 1;
        const int ox = -cw * dx, oy = -cw * dy;
        const int y0 = dy > 0 ? 0 : h - 1;
        const int pred = t - dx;   // predecessor in this sweep's scan order
        const bool has_pred = active && pred >= 0 && pred < nseg;
        load_row<C2, S>(P, dl, (long long)y0 * w + x0, n);
        load_row<C2, S>(C, dl, (long long)(y0 + dy) * w + x0, n);
#pragma unroll
        for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, oy));
        int g = 0;
        __syncthreads();   // the previous sweep's last pass may still read the slots
        if (active) {
            sh.guess[g][t] = dx > 0 ? seg_edge<C2, S, +1>(V, n) : seg_edge<C2, S, -1>(V, n);
            sh.edge[g][t] = dx > 0 ? seg_edge<C2, S, +1>(P, n) : seg_edge<C2, S, -1>(P, n);
        }
        __syncthreads();
        for (int j = 1; j < h; j++) {
            const int y = y0 + j * dy;
            const bool more = j + 1 < h;
            if (more) load_row<C2, S>(C, dl, (long long)(y + dy) * w + x0, n);
            // diagonal candidates from the previous row (P): own cells, then the predecessor's edge
            if (dx > 0) {
#pragma unroll
                for (int s = 1; s < S; s++) D[s] = add(P[s - 1], ox, oy);
            } else {
#pragma unroll
                for (int s = 0; s + 1 < S; s++) D[s] = add(P[s + 1], ox, oy);
            }
            if (has_pred) {
                const C2 e = add(sh.edge[g][pred], ox, oy);
                if (dx > 0) D[0] = e;
                else {
#pragma unroll
                    for (int s = 0; s < S; s++)
                        if (s == n - 1) D[s] = e;
                }
            }
            const C2 in0 = has_pred ? sh.guess[g][pred] : V[0];
            auto post = [&](const C2 (&X)[S]) {
                if (!active) return;
                if (dx > 0) {
                    sh.edge[g ^ 1][t] = seg_edge<C2, S, +1>(X, n);
                    if (more) sh.guess[g ^ 1][t] = closer(seg_edge<C2, S, +1>(C, n), add(seg_edge<C2, S, +1>(X, n), 0, oy));
                } else {
                    sh.edge[g ^ 1][t] = seg_edge<C2, S, -1>(X, n);
                    if (more) sh.guess[g ^ 1][t] = closer(seg_edge<C2, S, -1>(C, n), add(seg_edge<C2, S, -1>(X, n), 0, oy));
                }
            };
            if (dx > 0)
                row_pass<C2, S, true, +1>(R, V, t, nseg, n, cw, sh, D, in0, post);
            else
                row_pass<C2, S, true, -1>(R, V, t, nseg, n, cw, sh, D, in0, post);
            g ^= 1;
            store_row<C2, S>(dl, (long long)y * w + x0, R, n);
#pragma unroll
            for (int s = 0; s < S; s++) {
                P[s] = R[s];
                if (more) V[s] = closer(C[s], add(P[s], 0, oy));
            }
        }
    }
}

// ------------------------------------------------------------- FastSweep 3D ----

template <int S>
__global__ void __launch_bounds__(256) k_fastsweep3(int16_t* __restrict__ dl, int w, int h, int d, int cw, int sweep,
                                                    int* __restrict__ flags, int* __restrict__ counter,
                                                    const int* __restrict__ diag_start, int* __restrict__ err,
                                                    int epoch, int wait_epoch, unsigned wait_limit)
{
    __shared__ ScanShared<C3> sh;
    __shared__ long long s_item;
    __shared__ int s_c;
    const int t = threadIdx.x;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    const long long plane = (long long)w * h;
    const int dx = (sweep & 1) ? -1 : 1, dy = (sweep & 2) ? -1 : 1, dz = (sweep & 4) ? -1 : 1;
    const int oy = -cw * dy, oz = -cw * dz;
    const int yb = dy > 0 ? 0 : h - 1, zb = dz > 0 ? 0 : d - 1;
    const int H = h - 1, Dd = d - 1;
    const long long total = (long long)H * Dd;
    const int pred = t - dx;
    const bool has_pred = active && pred >= 0 && pred < nseg;
    C3 C[S], Zp[S], Yp[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) C[s] = Zp[s] = Yp[s] = V[s] = R[s] = D[s] = C3{0, 0, 0};

    // anti-diagonal c = jj + kk (jj: rows after the first, kk: slices after
    // the first) of the item: the last c with diag_start[c] <= item.  A CTA
    // claims items in increasing order, so its c only moves forward (thread 0
    // keeps it; a few cached loads per item instead of a binary search).  A
    // row is claimed only when the CTA is free to run it: claiming the next
    // one early parks rows of the wavefront behind another row's work
    // (measured 15.2 -> 24.0 ms at 256^3).
    int c_cur = 2;
    for (;;) {
        if (t == 0) {
            const long long it = atomicAdd(counter, 1);
            if (it < total)
                while (c_cur < H + Dd && diag_start[c_cur + 1] <= it) c_cur++;
            s_item = it;
            s_c = c_cur;
        }
        __syncthreads();
        const long long item = s_item;
        const int c = s_c;
        __syncthreads();
        if (item >= total) break;
        const int jj = max(1, c - Dd) + (int)(item - diag_start[c]);
        const int kk = c - jj;
        const int y = yb + jj * dy, z = zb + kk * dz;
        const int yprev = y - dy, zprev = z - dz;

        if (t == 0) {
            // wait (bounded) until both neighbour rows of this sweep are done
            const int* fa = jj > 1 ? flags + (long long)z * h + yprev : nullptr;
            const int* fb = kk > 1 ? flags + (long long)zprev * h + y : nullptr;
            // (wait_epoch is epoch except under a test hook that makes it unreachable)
            for (unsigned it = 0;; it++) {
                bool ok = (!fa || *((volatile const int*)fa) >= wait_epoch) &&
                          (!fb || *((volatile const int*)fb) >= wait_epoch);
                if (ok) break;
                if (it >= wait_limit) { atomicExch(err, 1); break; }
                __nanosleep(128);
            }
            __threadfence();
        }
        __syncthreads();

        const long long rb = z * plane + (long long)y * w + x0;
        const long long zb_ = (long long)zprev * plane + (long long)y * w + x0;
        const long long yb_ = z * plane + (long long)yprev * w + x0;
#pragma unroll
        for (int s = 0; s < S; s++)
            if (s < n) {
                C[s] = cell_load_cg(dl, rb + s);
                Zp[s] = cell_load_cg(dl, zb_ + s);
                Yp[s] = cell_load_cg(dl, yb_ + s);
                V[s] = closer(closer(C[s], add(Zp[s], 0, 0, oz)), add(Yp[s], 0, oy, 0));
            }
        if (active) sh.guess[0][t] = dx > 0 ? seg_edge<C3, S, +1>(V, n) : seg_edge<C3, S, -1>(V, n);
        __syncthreads();
        const C3 in0 = has_pred ? sh.guess[0][pred] : V[0];
        auto nopost = [](const C3 (&)[S]) {};
        if (dx > 0)
            row_pass<C3, S, false, +1>(R, V, t, nseg, n, cw, sh, D, in0, nopost);
        else
            row_pass<C3, S, false, -1>(R, V, t, nseg, n, cw, sh, D, in0, nopost);
        store_row<C3, S>(dl, rb, R, n);
        __threadfence();
        __syncthreads();
        if (t == 0) atomicExch(flags + (long long)z * h + y, epoch);
    }
}

// Slice pipeline (the default): a CTA claims a slice kk (in sweep order,
// from an atomic counter) and walks its rows jj = 1 .. H in order, so the
// row before (y - dy, same slice) is the CTA's own previous result, kept in
// registers; only the slice before (z - dz, same row) comes from another
// CTA, through its per-row flag.  Along y a step costs one row's work, along
// z one row's work plus the hand-over (the producer's fence and flag, the
// poll, the load), where the anti-diagonal wavefront above pays the
// hand-over on every step (256^3 shapes: 11.7 against 15.2 ms).  A slice is
// claimed only by a running CTA and waits only on the slice claimed before
// it, so the earliest unfinished slice always proceeds.  A row's own cells
// are written by no other CTA of the sweep, so they are loaded before the
// wait (loading the next row's during the hand-over measured 3 % slower).
template <int S>
__global__ void __launch_bounds__(256) k_fastsweep3_slices(int16_t* __restrict__ dl, int w, int h, int d, int cw,
                                                           int sweep, int* __restrict__ flags,
                                                           int* __restrict__ counter, int* __restrict__ err,
                                                           int epoch, int wait_epoch, unsigned wait_limit)
{
    __shared__ ScanShared<C3> sh;
    __shared__ int s_slice;
    const int t = threadIdx.x;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    const long long plane = (long long)w * h;
    const int dx = (sweep & 1) ? -1 : 1, dy = (sweep & 2) ? -1 : 1, dz = (sweep & 4) ? -1 : 1;
    const int oy = -cw * dy, oz = -cw * dz;
    const int yb = dy > 0 ? 0 : h - 1, zb = dz > 0 ? 0 : d - 1;
    const int H = h - 1, Dd = d - 1;
    const int pred = t - dx;
    const bool has_pred = active && pred >= 0 && pred < nseg;
    C3 C[S], Zp[S], Yp[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) C[s] = Zp[s] = Yp[s] = V[s] = R[s] = D[s] = C3{0, 0, 0};

    for (;;) {
        if (t == 0) s_slice = atomicAdd(counter, 1) + 1;
        __syncthreads();
        const int kk = s_slice;
        __syncthreads();
        if (kk > Dd) break;
        const int z = zb + kk * dz, zprev = z - dz;
        // the slice's first row is not updated by the sweep (:2208, :2214 start at 1)
#pragma unroll
        for (int s = 0; s < S; s++)
            if (s < n) Yp[s] = cell_load_cg(dl, z * plane + (long long)yb * w + x0 + s);
        for (int jj = 1; jj <= H; jj++) {
            const int y = yb + jj * dy;
            const long long rb = z * plane + (long long)y * w + x0;
#pragma unroll
            for (int s = 0; s < S; s++)
                if (s < n) C[s] = cell_load_cg(dl, rb + s);
            if (kk > 1 && t == 0) {
                // wait (bounded) until the slice before has done this row; the
                // poll is an acquire load, which with the barrier after it
                // orders the CTA's loads of that row after the producer's
                // stores (wait_epoch is epoch except under a test hook that
                // makes it unreachable)
                const int* fb = flags + (long long)zprev * h + y;
                for (unsigned it = 0;; it++) {
                    int f;
                    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(f) : "l"(fb) : "memory");
                    if (f >= wait_epoch) break;
                    if (it >= wait_limit) {
                        atomicExch(err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __syncthreads();
            const long long zb_ = (long long)zprev * plane + (long long)y * w + x0;
#pragma unroll
            for (int s = 0; s < S; s++)
                if (s < n) {
                    Zp[s] = cell_load_cg(dl, zb_ + s);
                    V[s] = closer(closer(C[s], add(Zp[s], 0, 0, oz)), add(Yp[s], 0, oy, 0));
                }
            if (active) sh.guess[0][t] = dx > 0 ? seg_edge<C3, S, +1>(V, n) : seg_edge<C3, S, -1>(V, n);
            __syncthreads();
            const C3 in0 = has_pred ? sh.guess[0][pred] : V[0];
            auto nopost = [](const C3 (&)[S]) {};
            if (dx > 0)
                row_pass<C3, S, false, +1>(R, V, t, nseg, n, cw, sh, D, in0, nopost);
            else
                row_pass<C3, S, false, -1>(R, V, t, nseg, n, cw, sh, D, in0, nopost);
            store_row<C3, S>(dl, rb, R, n);
#pragma unroll
            for (int s = 0; s < S; s++) Yp[s] = R[s];   // the next row's y neighbour
            // publish the row: after the barrier one thread's fence orders the
            // whole CTA's stores before the flag (the pattern of a grid
            // barrier); a thread of the second warp does it, so that thread 0
            // polls for the next row meanwhile and no other thread waits on a fence
            __syncthreads();
            if (t == (blockDim.x > 32 ? 32 : 0)) {
                __threadfence();
                atomicExch(flags + (long long)z * h + y, epoch);
            }
        }
    }
}

// ------------------------------------------------------- single-warp engines ----
// Rows of at most 32*S cells: one warp per image (or volume), every exchange a
// shuffle, no shared memory and no CTA barrier (row_pass_warp).  Same steps
// and candidate order as the CTA engines above.

template <int S>
__device__ __forceinline__ void danielsson2_warp(uint32_t* __restrict__ dl, int w, int h, int cw)
{
    const int lane = threadIdx.x & 31;
    const int nseg = (w + S - 1) / S;
    const bool active = lane < nseg;
    const int n = active ? min(S, w - lane * S) : 0;
    const long long x0 = (long long)lane * S;
    if (h < 2) return;
    const int steps = 2 * (h - 1);
    auto row_of = [&](int i) { return i < h - 1 ? i + 1 : 2 * h - 3 - i; };
    auto dy_of = [&](int i) { return i < h - 1 ? -cw : cw; };
    C2 P[S], C[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = V[s] = R[s] = D[s] = C2{0, 0};
    load_row<C2, S>(P, dl, x0, n);
    load_row<C2, S>(C, dl, (long long)row_of(0) * w + x0, n);
#pragma unroll
    for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, dy_of(0)));
    for (int i = 0; i < steps; i++) {
        const int y = row_of(i);
        const bool more = i + 1 < steps;
        if (more) load_row<C2, S>(C, dl, (long long)row_of(i + 1) * w + x0, n);
        row_pass_warp<C2, S, false, +1>(R, V, lane, nseg, n, cw, D, warp_round0_input<C2, S, +1>(V, n, lane));
        row_pass_warp<C2, S, false, -1>(P, R, lane, nseg, n, cw, D, warp_round0_input<C2, S, -1>(R, n, lane));
        store_row<C2, S>(dl, (long long)y * w + x0, P, n);
        if (more) {
            const int dyn = dy_of(i + 1);
#pragma unroll
            for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, dyn));
        }
    }
}

template <int S>
__device__ __forceinline__ void danielsson3_warp(int16_t* __restrict__ dl, int w, int h, int d, int cw)
{
    const int lane = threadIdx.x & 31;
    const int nseg = (w + S - 1) / S;
    const bool active = lane < nseg;
    const int n = active ? min(S, w - lane * S) : 0;
    const long long x0 = (long long)lane * S;
    const long long plane = (long long)w * h;
    const int steps = 2 * (h - 1);
    auto row_of = [&](int i) { return i < h - 1 ? i + 1 : 2 * h - 3 - i; };
    auto dy_of = [&](int i) { return i < h - 1 ? -cw : cw; };
    C3 P[S], C[S], Q[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = Q[s] = V[s] = R[s] = D[s] = C3{0, 0, 0};
    for (int pass = 0; pass < 2; pass++) {
        const int dz = pass == 0 ? -cw : +cw;
        for (int k = 1; k < d; k++) {
            const int z = pass == 0 ? k : d - 1 - k;
            const int zp = pass == 0 ? z - 1 : z + 1;
            const long long sb = z * plane, pb = (long long)zp * plane;
            load_row<C3, S>(C, dl, sb + x0, n);
            load_row<C3, S>(Q, dl, pb + x0, n);
#pragma unroll
            for (int s = 0; s < S; s++) P[s] = closer(C[s], add(Q[s], 0, 0, dz));
            store_row<C3, S>(dl, sb + x0, P, n);
            if (h < 2) continue;
            load_row<C3, S>(C, dl, sb + (long long)w + x0, n);
            load_row<C3, S>(Q, dl, pb + (long long)w + x0, n);
#pragma unroll
            for (int s = 0; s < S; s++) V[s] = closer(closer(C[s], add(Q[s], 0, 0, dz)), add(P[s], 0, -cw, 0));
            for (int i = 0; i < steps; i++) {
                const int y = row_of(i);
                const bool more = i + 1 < steps;
                const bool next_down = more && i + 1 < h - 1;
                if (more) {
                    const long long off = (long long)row_of(i + 1) * w + x0;
                    load_row<C3, S>(C, dl, sb + off, n);
                    if (next_down) load_row<C3, S>(Q, dl, pb + off, n);
                }
                row_pass_warp<C3, S, false, +1>(R, V, lane, nseg, n, cw, D, warp_round0_input<C3, S, +1>(V, n, lane));
                row_pass_warp<C3, S, false, -1>(P, R, lane, nseg, n, cw, D, warp_round0_input<C3, S, -1>(R, n, lane));
                store_row<C3, S>(dl, sb + (long long)y * w + x0, P, n);
                if (more) {
                    const int dyn = dy_of(i + 1);
#pragma unroll
                    for (int s = 0; s < S; s++) {
                        C3 c = next_down ? closer(C[s], add(Q[s], 0, 0, dz)) : C[s];
                        V[s] = closer(c, add(P[s], 0, dyn, 0));
                    }
                }
            }
        }
    }
}

template <int S>
__global__ void __launch_bounds__(32) k_danielsson2_w(uint32_t* __restrict__ dl, int w, int h, int cw)
{
    danielsson2_warp<S>(dl, w, h, cw);
}

template <int S>
__global__ void __launch_bounds__(32) k_danielsson3_w(int16_t* __restrict__ dl, int w, int h, int d, int cw)
{
    danielsson3_warp<S>(dl, w, h, d, cw);
}

template <int S>
__global__ void __launch_bounds__(32) k_fastsweep2_w(uint32_t* __restrict__ dl, int w, int h, int cw)
{
    const int lane = threadIdx.x & 31;
    const int nseg = (w + S - 1) / S;
    const bool active = lane < nseg;
    const int n = active ? min(S, w - lane * S) : 0;
    const long long x0 = (long long)lane * S;
    C2 P[S], C[S], V[S], R[S], D[S];
#pragma unroll
    for (int s = 0; s < S; s++) P[s] = C[s] = V[s] = R[s] = D[s] = C2{0, 0};
    if (h < 2) return;
    for (int sweep = 0; sweep < 4; sweep++) {
        const int dx = (sweep & 1) ? -1 : 1, dy = (sweep & 2) ? -1 : 1;
        const int ox = -cw * dx, oy = -cw * dy;
        const int y0 = dy > 0 ? 0 : h - 1;
        const int pred = lane - dx;
        const bool has_pred = active && pred >= 0 && pred < nseg;
        const int src = pred < 0 ? 0 : (pred > 31 ? 31 : pred);
        load_row<C2, S>(P, dl, (long long)y0 * w + x0, n);
        load_row<C2, S>(C, dl, (long long)(y0 + dy) * w + x0, n);
#pragma unroll
        for (int s = 0; s < S; s++) V[s] = closer(C[s], add(P[s], 0, oy));
        for (int j = 1; j < h; j++) {
            const int y = y0 + j * dy;
            const bool more = j + 1 < h;
            if (more) load_row<C2, S>(C, dl, (long long)(y + dy) * w + x0, n);
            // diagonal candidates from the previous row: own cells, then the predecessor's edge
            C2 e;
            if (dx > 0) {
#pragma unroll
                for (int s = 1; s < S; s++) D[s] = add(P[s - 1], ox, oy);
                e = shfl_cell(0xFFFFFFFFu, seg_edge<C2, S, +1>(P, n), src);
            } else {
#pragma unroll
                for (int s = 0; s + 1 < S; s++) D[s] = add(P[s + 1], ox, oy);
                e = shfl_cell(0xFFFFFFFFu, seg_edge<C2, S, -1>(P, n), src);
            }
            if (has_pred) {
                e = add(e, ox, oy);
                if (dx > 0) D[0] = e;
                else {
#pragma unroll
                    for (int s = 0; s < S; s++)
                        if (s == n - 1) D[s] = e;
                }
            }
            if (dx > 0)
                row_pass_warp<C2, S, true, +1>(R, V, lane, nseg, n, cw, D, warp_round0_input<C2, S, +1>(V, n, lane));
            else
                row_pass_warp<C2, S, true, -1>(R, V, lane, nseg, n, cw, D, warp_round0_input<C2, S, -1>(V, n, lane));
            store_row<C2, S>(dl, (long long)y * w + x0, R, n);
#pragma unroll
            for (int s = 0; s < S; s++) {
                P[s] = R[s];
                if (more) V[s] = closer(C[s], add(P[s], 0, oy));
            }
        }
    }
}

// --------------------------------------------------------------- launchers ----

// cells per thread: aim for at most 256 threads (fewer warps at every barrier),
// allow up to max_threads for wide rows; 0 when the row is too wide
static int pick_s(int w, int max_threads)
{
    const int options[] = {1, 2, 4, 8};
    for (int s : options)
        if ((w + s - 1) / s <= 256 && (w + s - 1) / s <= max_threads) return s;
    for (int s : options)
        if ((w + s - 1) / s <= max_threads) return s;
    return 0;
}

// the tuned cells-per-thread for this family and width, if it fits
static int tuned_s(int kind, int w, int max_threads)
{
    const int v = tune_get(kind, w);
    if ((v == 1 || v == 2 || v == 4 || v == 8) && (w + v - 1) / v <= max_threads) return v;
    return pick_s(w, max_threads);
}

static int threads_for(int w, int s)
{
    int n = (w + s - 1) / s;
    return ((n + 31) / 32) * 32;
}

// The single-warp engines take rows up to 32 * 16 cells (2D) / 32 * 8 (3D).
// Tuning value kWarpEngine selects them; 1/2/4/8 select the CTA engine with
// that many cells per thread; 0 (untuned) picks the warp engine when it fits.
constexpr int kWarpEngine = 32;

static int warp_s(int w, int max_s)
{
    for (int s = 1; s <= max_s; s *= 2)
        if (32 * s >= w) return s;
    return 0;
}

void launch_danielsson(int dim, void* deltas, int w, int h, int d, int cw, cudaStream_t st)
{
    const int kind = dim == 2 ? kTuneDan2 : kTuneDan3;
    const int tv = tune_get(kind, w);
    const int ws = warp_s(w, dim == 2 ? 16 : 8);
    ProfScope ps("danielsson", st);
    if (ws && (tv == kWarpEngine || tv == 0)) {
#define DOL_DANW_CASE(SV)                                                                             \
    case SV:                                                                                          \
        if (dim == 2)                                                                                 \
            k_danielsson2_w<SV><<<1, 32, 0, st>>>(static_cast<uint32_t*>(deltas), w, h, cw);         \
        else                                                                                          \
            k_danielsson3_w<(SV > 8 ? 8 : SV)><<<1, 32, 0, st>>>(static_cast<int16_t*>(deltas), w, h, d, cw); \
        return;
        switch (ws) {
            DOL_DANW_CASE(1)
            DOL_DANW_CASE(2)
            DOL_DANW_CASE(4)
            DOL_DANW_CASE(8)
            DOL_DANW_CASE(16)
            default: break;
        }
#undef DOL_DANW_CASE
    }
    const int s = tuned_s(kind, w, 512);
    const int T = threads_for(w, s);
#define DOL_DAN_CASE(SV)                                                                              \
    case SV:                                                                                          \
        if (dim == 2)                                                                                 \
            k_danielsson2<SV><<<1, T, 0, st>>>(static_cast<uint32_t*>(deltas), w, h, cw);            \
        else                                                                                          \
            k_danielsson3<SV><<<1, T, 0, st>>>(static_cast<int16_t*>(deltas), w, h, d, cw);          \
        break;
    switch (s) {
        DOL_DAN_CASE(1)
        DOL_DAN_CASE(2)
        DOL_DAN_CASE(4)
        DOL_DAN_CASE(8)
        default: break;
    }
#undef DOL_DAN_CASE
}

void launch_fastsweep_2d(void* deltas, int w, int h, int cw, cudaStream_t st)
{
    const int tv = tune_get(kTuneFs2, w);
    const int ws = warp_s(w, 16);
    ProfScope ps("fastsweep_2d", st);
    if (ws && (tv == kWarpEngine || tv == 0)) {
#define DOL_FSW_CASE(SV)                                                                              \
    case SV:                                                                                          \
        k_fastsweep2_w<SV><<<1, 32, 0, st>>>(static_cast<uint32_t*>(deltas), w, h, cw);              \
        return;
        switch (ws) {
            DOL_FSW_CASE(1)
            DOL_FSW_CASE(2)
            DOL_FSW_CASE(4)
            DOL_FSW_CASE(8)
            DOL_FSW_CASE(16)
            default: break;
        }
#undef DOL_FSW_CASE
    }
    const int s = tuned_s(kTuneFs2, w, 512);
    const int T = threads_for(w, s);
#define DOL_FS_CASE(SV)                                                                                      \
    case SV:                                                                                                 \
        k_fastsweep2<SV><<<1, T, 0, st>>>(static_cast<uint32_t*>(deltas), w, h, cw);                         \
        break;
    switch (s) {
        DOL_FS_CASE(1)
        DOL_FS_CASE(2)
        DOL_FS_CASE(4)
        DOL_FS_CASE(8)
        default: break;
    }
#undef DOL_FS_CASE
}

size_t fastsweep3_workspace_bytes(int w, int h, int d)
{
    (void)w;
    size_t flags = (size_t)h * d * sizeof(int);
    size_t diag = (size_t)(h + d + 2) * sizeof(int);
    return ((flags + 255) & ~(size_t)255) + ((diag + 255) & ~(size_t)255) + 256;
}

void launch_fastsweep_3d(void* deltas, int w, int h, int d, int cw, void* ws, int* err, cudaStream_t st)
{
    if (h < 2 || d < 2) return;   // no row is ever updated (:2208, :2214 start at 1)
    char* p = static_cast<char*>(ws);
    int* flags = reinterpret_cast<int*>(p);
    p += (((size_t)h * d * sizeof(int)) + 255) & ~(size_t)255;
    int* diag = reinterpret_cast<int*>(p);
    p += (((size_t)(h + d + 2) * sizeof(int)) + 255) & ~(size_t)255;
    int* counters = reinterpret_cast<int*>(p);   // 8 ints

    // anti-diagonal starts: rows jj in [1, h-1], kk in [1, d-1], c = jj + kk
    const int H = h - 1, Dd = d - 1;
    static thread_local int* host_diag = nullptr;
    static thread_local size_t host_diag_n = 0;
    size_t nd = (size_t)(H + Dd + 2);
    if (host_diag_n < nd) {
        if (host_diag) cudaFreeHost(host_diag);
        cudaMallocHost(&host_diag, nd * sizeof(int));
        host_diag_n = nd;
    }
    long long acc = 0;
    for (int c = 0; c < (int)nd; c++) {
        host_diag[c] = (int)acc;
        if (c >= 2 && c <= H + Dd) {
            int lo = c - Dd > 1 ? c - Dd : 1, hi = c - 1 < H ? c - 1 : H;
            if (hi >= lo) acc += hi - lo + 1;
        }
    }
    cudaMemcpyAsync(diag, host_diag, nd * sizeof(int), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(flags, 0, (size_t)h * d * sizeof(int), st);
    cudaMemsetAsync(counters, 0, 8 * sizeof(int), st);

    // cells per thread: tuned, else rows of at most 128 threads (more CTAs
    // per SM along the wavefront; 256^3 shapes: 15.1 ms at 128 threads, 22.0
    // at 256), else at most 256
    int s = tune_get(kTuneFs3, w);
    const bool wavefront = s < 0;   // negative tuned values: the anti-diagonal wavefront with -s cells per thread
    if (wavefront) s = -s;
    if (!((s == 1 || s == 2 || s == 4 || s == 8) && (w + s - 1) / s <= 256)) {
        s = pick_s(w, 128);
        if (!s) s = pick_s(w, 256);
    }
    const int T = threads_for(w, s);
    const WaitHooks hooks = wait_hooks();
    ProfScope ps("fastsweep_3d", st);
#define DOL_FS3_CASE(SV)                                                                                     \
    case SV: {                                                                                               \
        if (!wavefront) {                                                                                    \
            int per_sm = 0;                                                                                  \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fastsweep3_slices<SV>, T, 0);           \
            if (per_sm < 1) per_sm = 1;                                                                      \
            long long grid = (long long)per_sm * g_num_sms;                                                  \
            if (grid > Dd) grid = Dd;                                                                        \
            for (int sw = 0; sw < 8; sw++)                                                                   \
                k_fastsweep3_slices<SV><<<(int)grid, T, 0, st>>>(static_cast<int16_t*>(deltas), w, h, d, cw,  \
                                                                 sw, flags, counters + sw, err, sw + 1,       \
                                                                 sw == hooks.stall_sweep ? INT_MAX : sw + 1,  \
                                                                 hooks.limit);                                \
            break;                                                                                           \
        }                                                                                                    \
        int per_sm = 0;                                                                                      \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fastsweep3<SV>, T, 0);                      \
        if (per_sm < 1) per_sm = 1;                                                                          \
        long long rows = (long long)H * Dd;                                                                  \
        long long grid = (long long)per_sm * g_num_sms;                                                      \
        if (grid > rows) grid = rows;                                                                        \
        for (int sw = 0; sw < 8; sw++)                                                                       \
            k_fastsweep3<SV><<<(int)grid, T, 0, st>>>(static_cast<int16_t*>(deltas), w, h, d, cw, sw, flags,  \
                                                      counters + sw, diag, err, sw + 1,                       \
                                                      sw == hooks.stall_sweep ? INT_MAX : sw + 1,             \
                                                      hooks.limit);                                           \
    } break;
    switch (s) {
        DOL_FS3_CASE(1)
        DOL_FS3_CASE(2)
        DOL_FS3_CASE(4)
        DOL_FS3_CASE(8)
        default: break;
    }
#undef DOL_FS3_CASE
}

}  // namespace dolk

// ------------------------------------------------------------- batched SDF ----
// Thousands of independent masks and volumes in one persistent launch: each
// CTA pulls the next item (largest first) from an atomic counter and runs the
// whole signed pipeline on it -- border initialisation, Danielsson with cw = 2,
// signed distances -- with the same per-CTA code as the single-item kernels,
// so every item's output is bit-identical to a per-item call.
#include "border.cuh"

namespace dolk {

struct BatchItemDev {
    int w, h, d, pad;
    long long mask_off;    // words
    long long delta_off;   // bytes
    long long dist_off;    // floats, < 0: none
};

__device__ __forceinline__ void border2_cta(const uint32_t* mask, uint32_t* dl, int w, int h)
{
    const int ws = words_per_row(w);
    for (long long wid = threadIdx.x; wid < (long long)ws * h; wid += blockDim.x) {
        const int y = (int)(wid / ws), k = (int)(wid - (long long)y * ws);
        Planes2 p = border2_word(w, h, mask, y, k);
        const int n = min(32, w - 32 * k);
        uint32_t* row = dl + (long long)y * w + 32 * k;
        for (int b = 0; b < n; b++) row[b] = pack2(decode2(p, b));
    }
}

__device__ __forceinline__ void border3_cta(const uint32_t* mask, int16_t* dl, int w, int h, int d)
{
    const int ws = words_per_row(w);
    const long long words = (long long)ws * h * d;
    for (long long wid = threadIdx.x; wid < words; wid += blockDim.x) {
        const long long row = wid / ws;
        const int k = (int)(wid - row * ws);
        const int z = (int)(row / h), y = (int)(row - (long long)z * h);
        Planes3 p = border3_word(w, h, d, mask, z, y, k);
        const int n = min(32, w - 32 * k);
        for (int b = 0; b < n; b++) cell_store(dl, row * w + 32 * k + b, decode3(p, b));
    }
}

template <class Cell, class P>
__device__ __forceinline__ void signed_dist_cta(const uint32_t* mask, const P* dl, float* out, int w, long long rows)
{
    const int ws = words_per_row(w);
    for (long long i = threadIdx.x; i < rows * w; i += blockDim.x) {
        const long long row = i / w;
        const int x = (int)(i - row * w);
        float r = __fdiv_rn(sqrtf((float)len(cell_load(dl, i))), 2.0f);
        if ((mask[row * ws + (x >> 5)] >> (x & 31)) & 1u) r = -r;
        out[i] = r;
    }
}

// warp-cooperative pieces for items whose rows fit one warp
__device__ __forceinline__ void border2_warp(const uint32_t* mask, uint32_t* dl, int w, int h)
{
    const int lane = threadIdx.x & 31;
    const int ws = words_per_row(w);
    for (long long wid = lane; wid < (long long)ws * h; wid += 32) {
        const int y = (int)(wid / ws), k = (int)(wid - (long long)y * ws);
        Planes2 p = border2_word(w, h, mask, y, k);
        const int n = min(32, w - 32 * k);
        uint32_t* row = dl + (long long)y * w + 32 * k;
        for (int b = 0; b < n; b++) row[b] = pack2(decode2(p, b));
    }
}

__device__ __forceinline__ void border3_warp(const uint32_t* mask, int16_t* dl, int w, int h, int d)
{
    const int lane = threadIdx.x & 31;
    const int ws = words_per_row(w);
    const long long words = (long long)ws * h * d;
    for (long long wid = lane; wid < words; wid += 32) {
        const long long row = wid / ws;
        const int k = (int)(wid - row * ws);
        const int z = (int)(row / h), y = (int)(row - (long long)z * h);
        Planes3 p = border3_word(w, h, d, mask, z, y, k);
        const int n = min(32, w - 32 * k);
        for (int b = 0; b < n; b++) cell_store(dl, row * w + 32 * k + b, decode3(p, b));
    }
}

template <class Cell, class P>
__device__ __forceinline__ void signed_dist_warp(const uint32_t* mask, const P* dl, float* out, int w, long long rows)
{
    const int lane = threadIdx.x & 31;
    const int ws = words_per_row(w);
    for (long long i = lane; i < rows * w; i += 32) {
        const long long row = i / w;
        const int x = (int)(i - row * w);
        float r = __fdiv_rn(sqrtf((float)len(cell_load(dl, i))), 2.0f);
        if ((mask[row * ws + (x >> 5)] >> (x & 31)) & 1u) r = -r;
        out[i] = r;
    }
}

// an item processed by one warp: rows of at most 256 cells
__device__ __noinline__ void batch_item_warp(const BatchItemDev& b, const uint32_t* masks, unsigned char* deltas,
                                             float* dist)
{
    const uint32_t* m = masks + b.mask_off;
    if (b.d <= 1) {
        uint32_t* dl = reinterpret_cast<uint32_t*>(deltas + b.delta_off);
        border2_warp(m, dl, b.w, b.h);
        __syncwarp();
        if (b.w <= 64) danielsson2_warp<2>(dl, b.w, b.h, 2);
        else if (b.w <= 128) danielsson2_warp<4>(dl, b.w, b.h, 2);
        else danielsson2_warp<8>(dl, b.w, b.h, 2);
        __syncwarp();
        if (dist && b.dist_off >= 0) signed_dist_warp<C2>(m, dl, dist + b.dist_off, b.w, b.h);
    } else {
        int16_t* dl = reinterpret_cast<int16_t*>(deltas + b.delta_off);
        border3_warp(m, dl, b.w, b.h, b.d);
        __syncwarp();
        if (b.w <= 64) danielsson3_warp<2>(dl, b.w, b.h, b.d, 2);
        else if (b.w <= 128) danielsson3_warp<4>(dl, b.w, b.h, b.d, 2);
        else danielsson3_warp<8>(dl, b.w, b.h, b.d, 2);
        __syncwarp();
        if (dist && b.dist_off >= 0) signed_dist_warp<C3>(m, dl, dist + b.dist_off, b.w, (long long)b.h * b.d);
    }
}

// Two queues.  Queue A (order[0 .. nv)) holds the volumes whose rows fit one
// warp (up to 256 cells), longest chain first; queue B (order[nv .. n)) the
// items with rows over 256 cells, then the narrow images.  A CTA takes queue A
// items while there are any: the whole CTA runs the volume's border init and
// its distances, while warp 0 alone runs the serial sweep with the
// single-warp engine (no CTA barriers in the chain; 1.5-2x faster than the
// CTA engine on rows this narrow).  Then it turns to queue B: items with wide
// rows take the whole CTA; the first narrow image it draws switches it to
// per-warp draining.  counter: [0] queue B, [1] queue A, [2] nv (written by
// dol_batch_prepare).
template <int S>
__global__ void __launch_bounds__(256) k_batch_sdf(const BatchItemDev* __restrict__ items, const int* __restrict__ order,
                                                   int n, const uint32_t* __restrict__ masks,
                                                   unsigned char* __restrict__ deltas, float* __restrict__ dist,
                                                   int* __restrict__ counter)
{
    __shared__ ScanShared<C3> sh3;   // the larger of the two; the 2D engine reuses its storage
    __shared__ int s_item;
    ScanShared<C2>& sh2 = *reinterpret_cast<ScanShared<C2>*>(&sh3);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nv = counter[2];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter + 1, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nv) break;
        const BatchItemDev b = items[order[it]];
        const uint32_t* m = masks + b.mask_off;
        int16_t* dl = reinterpret_cast<int16_t*>(deltas + b.delta_off);
        border3_cta(m, dl, b.w, b.h, b.d);
        __syncthreads();
        if (warp == 0) {
            if (b.w <= 64) danielsson3_warp<2>(dl, b.w, b.h, b.d, 2);
            else if (b.w <= 128) danielsson3_warp<4>(dl, b.w, b.h, b.d, 2);
            else danielsson3_warp<8>(dl, b.w, b.h, b.d, 2);
        }
        __syncthreads();
        if (dist && b.dist_off >= 0) signed_dist_cta<C3>(m, dl, dist + b.dist_off, b.w, (long long)b.h * b.d);
        __syncthreads();
    }
    for (;;) {
        if (threadIdx.x == 0) s_item = nv + atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= n) return;
        const BatchItemDev b = items[order[it]];
        if (b.w <= 256) {
            // narrow images from here on: warp 0 takes this item, every warp then drains the queue
            int mine = warp == 0 ? it : -1;
            for (;;) {
                if (mine < 0) {
                    int v = 0;
                    if (lane == 0) v = nv + atomicAdd(counter, 1);
                    mine = __shfl_sync(0xFFFFFFFFu, v, 0);
                    if (mine >= n) return;
                }
                batch_item_warp(items[order[mine]], masks, deltas, dist);
                mine = -1;
            }
        }
        const uint32_t* m = masks + b.mask_off;
        if (b.d <= 1) {
            uint32_t* dl = reinterpret_cast<uint32_t*>(deltas + b.delta_off);
            border2_cta(m, dl, b.w, b.h);
            __syncthreads();
            danielsson2_cta<S>(dl, b.w, b.h, 2, sh2);
            __syncthreads();
            if (dist && b.dist_off >= 0) signed_dist_cta<C2>(m, dl, dist + b.dist_off, b.w, b.h);
        } else {
            int16_t* dl = reinterpret_cast<int16_t*>(deltas + b.delta_off);
            border3_cta(m, dl, b.w, b.h, b.d);
            __syncthreads();
            danielsson3_cta<S>(dl, b.w, b.h, b.d, 2, sh3);
            __syncthreads();
            if (dist && b.dist_off >= 0) signed_dist_cta<C3>(m, dl, dist + b.dist_off, b.w, (long long)b.h * b.d);
        }
        __syncthreads();
    }
}

static_assert(sizeof(BatchItemDev) == 40, "batch item layout (dol_batch_item)");

void launch_batch_sdf(const void* items, const int* order, int n, const uint32_t* masks, void* deltas, float* dist,
                      int* counter, cudaStream_t st)
{
    ProfScope ps("batch_sdf", st);
    // rows up to 1024 cells: 4 cells x 256 threads, or 8 cells x 128 threads
    const bool eight = tune_get(kTuneBatch, 1024) == 8;
    const int threads = eight ? 128 : 256;
    int per_sm = 0;
    if (eight)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_sdf<8>, threads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_sdf<4>, threads, 0);
    if (per_sm < 1) per_sm = 1;
    int grid = per_sm * g_num_sms;
    if (grid > n) grid = n;
    if (grid < 1) grid = 1;
    cudaMemsetAsync(counter, 0, 2 * sizeof(int), st);   // the queue heads; counter[2] (nv) stays
    if (eight)
        k_batch_sdf<8><<<grid, threads, 0, st>>>(static_cast<const BatchItemDev*>(items), order, n, masks,
                                                 static_cast<unsigned char*>(deltas), dist, counter);
    else
        k_batch_sdf<4><<<grid, threads, 0, st>>>(static_cast<const BatchItemDev*>(items), order, n, masks,
                                                 static_cast<unsigned char*>(deltas), dist, counter);
}

}  // namespace dolk
