// k_dan_blocks.cu -- Danielsson (2D and 3D) as a fixed-point iteration over
// blocks of rows, bit-identical to the serial sweeps.
//
// The reference's Danielsson (DistanceOcclusionLib.cpp:702-778 2D,
// :2264-2394 3D) is one long chain: every row needs the previous row, every
// slice the previous slice after its full 2D sweep.  Cut each sweep phase (the
// 2D image; each z direction of a volume) into blocks of R rows of one slice.
// A block runs the reference's steps over its rows -- z pull from the
// previous slice, then rows y0..y1-1 going down, then y1-1..y0 going up --
// from three inputs that other blocks produce:
//
//   Z  the previous slice's rows y0..y1-1 after its sweep  (block (z-dir, c))
//   D  row y0-1 after the down sweep                         (block (z, c-1))
//   U  row y1 after the up sweep                             (block (z, c+1))
//
// Every block starts from guesses (the phase input's own rows), all blocks
// run in parallel, and each round recomputes exactly the blocks whose inputs
// changed in the round before.  At the stop every block's inputs equal its
// producers' outputs, so by induction along the serial order (split into down
// and up halves it is acyclic: down(c) needs down(c-1); up(c) needs up(c+1)
// and down(c)) every output is the serial one.  Round r finalises at least
// one more half-block of the chain, so the iteration ends; in practice after
// about as many rounds as the longest distance in cells (a seed's influence
// crosses one slice per round), whatever R is.
//
// Outputs alternate between two version buffers per block, so a round reads
// only the previous round's outputs; a block's version flips when its new
// output differs from the old one.  One cooperative launch runs all rounds:
// blocks are taken from a work list, a block that changed queues its
// dependents for the next round, and two grid barriers (bounded waits) close
// each round.
#include "kernels.h"
#include "scan.cuh"

namespace dolk {

constexpr int kBlkThreads = 256;   // the widest CTA (rows up to 8 x 256 cells)

template <class Cell>
struct CellIO;
template <>
struct CellIO<C2> {
    using P = uint32_t;
    static constexpr int kWords = 1;
    static __device__ __forceinline__ C2 ld(const P* p, long long i) { return unpack2(__ldcg(p + i)); }
    static __device__ __forceinline__ void st(P* p, long long i, C2 c) { p[i] = pack2(c); }
};
template <>
struct CellIO<C3> {
    using P = int16_t;
    static constexpr int kWords = 3;
    static __device__ __forceinline__ C3 ld(const P* p, long long i)
    {
        const P* c = p + 3 * i;
        return C3{__ldcg(c), __ldcg(c + 1), __ldcg(c + 2)};
    }
    static __device__ __forceinline__ void st(P* p, long long i, C3 c)
    {
        P* o = p + 3 * i;
        o[0] = (P)c.x;
        o[1] = (P)c.y;
        o[2] = (P)c.z;
    }
};

DOL_HD C2 yshift(C2 c, int dy) { return add(c, 0, dy); }
DOL_HD C3 yshift(C3 c, int dy) { return add(c, 0, dy, 0); }

struct DanBlk {
    const void* A;         // phase input, unchanged during the phase
    void* V[2];            // output versions (cells, same layout as A)
    void* DB[2];           // per block and version: its last row after the down sweep
    uint8_t* lat;          // per block: version holding its output (2: none yet, the input's rows stand)
    uint8_t* chg;          // per block: change bits of its last computation
    int* stamp;            // per block: last round it was queued for
    int* wl[2];            // work lists by round parity
    unsigned* ctl;         // [0],[1] work-list sizes, [2] work counter, [3],[4] grid barrier, [5] rounds used
    int* err;
    int w, h, d, R, nc, cw;
    int dir;      // +1: slices zfirst, zfirst+1, ...; -1: downwards
    int zfirst;   // first slice of the phase's chain (the slice before it keeps its input)
    int nchain;   // slices in the chain (2D: 1)
    int Z;        // slices per block
    int nk;       // blocks along the chain: ceil(nchain / Z)
    int nblocks;  // nk * nc
    int max_rounds;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier for a cooperative launch (all CTAs resident).  The wait gives
// up after `limit_ns`, sets *err and returns false in every thread of the CTA.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, int* err, unsigned long long limit_ns)
{
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        volatile unsigned* vg = gen;
        const unsigned g = *vg;
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*vg == g) {
                __nanosleep(100);
                if (global_ns() - t0 > limit_ns) {
                    atomicExch(err, 2);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
    }
    return __syncthreads_and(ok);
}

// bits of DanBlk::chg
constexpr int kChgLast = 1;    // a row of the block's last slice changed  -> block (k+1, c)
constexpr int kChgFirst = 2;   // row y0 of some slice changed             -> block (k, c-1)
constexpr int kChgDown = 4;    // the down-sweep row y1-1 of some slice    -> block (k, c+1)
constexpr int kChgAny = 8;     // any output changed: the block's version flips

// One block: rows y0..y1-1 of Z consecutive slices (in the phase's order),
// T threads of S cells each.
template <class Cell, int kDim, int S, int T>
__device__ __forceinline__ void dan_block(const DanBlk& p, int b, ScanShared<Cell, T>& sh, int* s_chg)
{
    using IO = CellIO<Cell>;
    using P = typename IO::P;
    const int t = threadIdx.x;
    const int w = p.w, h = p.h, cw = p.cw;
    const int nseg = (w + S - 1) / S;
    const bool active = t < nseg;
    const int n = active ? min(S, w - t * S) : 0;
    const long long x0 = (long long)t * S;
    const int k = b / p.nc;
    const int c = b - k * p.nc;
    const int y0 = c * p.R, y1 = min(y0 + p.R, h), L = y1 - y0;
    const long long plane = (long long)w * h;
    const P* A = static_cast<const P*>(p.A);
    auto ver = [&](int v) -> const P* { return v == 2 ? A : static_cast<const P*>(p.V[v]); };
    const int vo = __ldcg(p.lat + b), vn = vo == 0 ? 1 : 0;
    const P* oldv = ver(vo);
    P* out = static_cast<P*>(p.V[vn]);
    // neighbour blocks' versions (fixed for the whole round)
    const int vd = c > 0 ? __ldcg(p.lat + b - 1) : 2;
    const int vu = y1 < h ? __ldcg(p.lat + b + 1) : 2;
    const int vz = (kDim == 3 && k > 0) ? __ldcg(p.lat + b - p.nc) : 2;
    const int dz = kDim == 3 ? -p.dir * cw : 0;
    const int pos0 = k * p.Z, nsl = min(p.Z, p.nchain - pos0);

    auto ldrow = [&](Cell (&dst)[S], const P* base, long long first) {
#pragma unroll
        for (int s = 0; s < S; s++)
            if (s < n) dst[s] = IO::ld(base, first + s);
    };
    auto strow = [&](P* base, long long first, const Cell (&src)[S]) {
#pragma unroll
        for (int s = 0; s < S; s++)
            if (s < n) IO::st(base, first + s, src[s]);
    };
    auto zpull = [&](Cell cc, Cell q) -> Cell {
        if constexpr (kDim == 3)
            return closer(cc, add(q, 0, 0, dz));
        else
            return cc;
    };

    Cell Pr[S], V[S], Rr[S], D[S], Cn[S], Qn[S];
#pragma unroll
    for (int s = 0; s < S; s++) Pr[s] = V[s] = Rr[s] = D[s] = Cn[s] = Qn[s] = Cell{};
    int bits = 0;
    int g = 0;

    for (int j = 0; j < nsl; j++) {
        const int z = p.zfirst + p.dir * (pos0 + j);
        const long long sb = (long long)z * plane;
        const bool last = j == nsl - 1;
        // the previous slice after its sweep: this block's own output, or the
        // block before in z (or the fixed slice, which keeps the input)
        const P* zin = nullptr;
        if (kDim == 3) zin = (j > 0 ? static_cast<const P*>(out) : ver(vz)) + IO::kWords * (sb - p.dir * plane);
        const long long dbi = ((long long)z * p.nc + c) * w;   // this slice's down-boundary row slot
        const P* gd = nullptr;   // row y0-1 after the down sweep
        if (c > 0)
            gd = vd == 2 ? A + IO::kWords * (sb + (long long)(y0 - 1) * w)
                         : static_cast<const P*>(p.DB[vd]) + IO::kWords * (dbi - w);
        const P* gu = nullptr;   // row y1 after the up sweep
        if (y1 < h) gu = ver(vu) + IO::kWords * (sb + (long long)y1 * w);
        const P* dbo = vo == 2 ? A + IO::kWords * (sb + (long long)(y1 - 1) * w)
                               : static_cast<const P*>(p.DB[vo]) + IO::kWords * dbi;
        P* dbn = static_cast<P*>(p.DB[vn]) + IO::kWords * dbi;

        // row y0 before its x passes
        ldrow(Cn, A, sb + (long long)y0 * w + x0);
        if (kDim == 3) ldrow(Qn, zin, (long long)y0 * w + x0);
#pragma unroll
        for (int s = 0; s < S; s++) V[s] = kDim == 3 ? zpull(Cn[s], Qn[s]) : Cn[s];
        if (gd) {
            ldrow(Qn, gd, x0);
#pragma unroll
            for (int s = 0; s < S; s++) V[s] = closer(V[s], yshift(Qn[s], -cw));
        }
        __syncthreads();   // the previous slice's last pass may still read the guess slots
        if (active) sh.guess[g][t] = seg_edge<Cell, S, +1>(V, n);
        __syncthreads();

        for (int i = 0; i < 2 * L; i++) {
            const bool down = i < L;
            const int y = down ? y0 + i : y1 - 1 - (i - L);
            const bool pass = down ? y > 0 : y < h - 1;
            const int nx = i + 1;                     // next step
            const bool more = nx < 2 * L;
            const bool nx_down = nx < L;
            const bool nx_turn = nx == L;             // first up step: base = this result, candidate = U
            const bool has_u = gu != nullptr;
            const long long rf = sb + (long long)y * w + x0;
            // the old output this step's result is compared with, loaded
            // before the passes so its latency hides behind them
            Cell O[S];
#pragma unroll
            for (int s = 0; s < S; s++) O[s] = Cell{};
            if (!down)
                ldrow(O, oldv, rf);
            else if (i == L - 1)
                ldrow(O, dbo, x0);
            // prefetch what the next step needs
            if (more) {
                if (nx_down) {
                    ldrow(Cn, A, sb + (long long)(y + 1) * w + x0);
                    if (kDim == 3) ldrow(Qn, zin, (long long)(y + 1) * w + x0);
                } else if (nx_turn) {
                    if (has_u) ldrow(Cn, gu, x0);
                } else {
                    ldrow(Cn, out, sb + (long long)(y - 1) * w + x0);   // its down-sweep result
                }
            }
            // the next step's row before its x passes, from this step's result X
            auto next_edge = [&](const Cell (&X)[S]) -> Cell {
                const Cell e = seg_edge<Cell, S, +1>(X, n);
                if (nx_down) {
                    const Cell cb = kDim == 3 ? zpull(seg_edge<Cell, S, +1>(Cn, n), seg_edge<Cell, S, +1>(Qn, n))
                                              : seg_edge<Cell, S, +1>(Cn, n);
                    return closer(cb, yshift(e, -cw));
                }
                if (nx_turn) return has_u ? closer(e, yshift(seg_edge<Cell, S, +1>(Cn, n), cw)) : e;
                return closer(seg_edge<Cell, S, +1>(Cn, n), yshift(e, cw));
            };
            if (pass) {
                const Cell in0 = (active && t > 0) ? sh.guess[g][t - 1] : V[0];
                row_pass<Cell, S, false, +1>(Rr, V, t, nseg, n, cw, sh, D, in0, [&](const Cell (&X)[S]) {
                    if (active) sh.guess[g ^ 1][t] = X[0];
                });
                g ^= 1;
                const Cell in1 = (active && t + 1 < nseg) ? sh.guess[g][t + 1] : Rr[0];
                row_pass<Cell, S, false, -1>(Pr, Rr, t, nseg, n, cw, sh, D, in1, [&](const Cell (&X)[S]) {
                    if (more && active) sh.guess[g ^ 1][t] = next_edge(X);
                });
                g ^= 1;
            } else {
#pragma unroll
                for (int s = 0; s < S; s++) Pr[s] = V[s];
                if (more && active) sh.guess[g][t] = next_edge(Pr);
                __syncthreads();
            }
            if (down) {
                strow(out, rf, Pr);
                if (i == L - 1) {
#pragma unroll
                    for (int s = 0; s < S; s++)
                        if (s < n && !same(O[s], Pr[s])) bits |= kChgDown | kChgAny;
                    strow(dbn, x0, Pr);
                }
            } else {
                bool diff = false;
#pragma unroll
                for (int s = 0; s < S; s++)
                    if (s < n && !same(O[s], Pr[s])) diff = true;
                if (diff) bits |= kChgAny | (last ? kChgLast : 0) | (y == y0 ? kChgFirst : 0);
                strow(out, rf, Pr);
            }
            if (more) {
                if (nx_down) {
#pragma unroll
                    for (int s = 0; s < S; s++) {
                        const Cell cb = kDim == 3 ? zpull(Cn[s], Qn[s]) : Cn[s];
                        V[s] = closer(cb, yshift(Pr[s], -cw));
                    }
                } else if (nx_turn) {
#pragma unroll
                    for (int s = 0; s < S; s++) V[s] = has_u ? closer(Pr[s], yshift(Cn[s], cw)) : Pr[s];
                } else {
#pragma unroll
                    for (int s = 0; s < S; s++) V[s] = closer(Cn[s], yshift(Pr[s], cw));
                }
            }
        }
    }
    if (bits) atomicOr(s_chg, bits);
    __syncthreads();
}

// T threads per CTA (a multiple of 32 covering the row's segments); the
// register budget allows 512 / T * ... CTAs: 128 registers a thread
template <class Cell, int kDim, int S, int T>
__global__ void __launch_bounds__(T, 512 / T) k_dan_blocks(DanBlk p)
{
    __shared__ ScanShared<Cell, T> sh;
    __shared__ int s_item, s_chg;
    const int t = threadIdx.x;
    const unsigned long long kLimit = 20ull * 1000 * 1000 * 1000;   // 20 s per barrier wait
    int round = 0;
    for (;; round++) {
        const int cur = round & 1;
        if (round >= p.max_rounds) {
            if (blockIdx.x == 0 && t == 0) atomicExch(p.err, 3);
            return;
        }
        const unsigned nwork = __ldcg(p.ctl + cur);
        const int* wl = p.wl[cur];
        int* wln = p.wl[cur ^ 1];
        for (;;) {
            if (t == 0) {
                s_item = (int)atomicAdd(p.ctl + 2, 1u);
                s_chg = 0;
            }
            __syncthreads();
            const unsigned it = (unsigned)s_item;
            if (it >= nwork) break;
            const int b = __ldcg(wl + it);
            dan_block<Cell, kDim, S, T>(p, b, sh, &s_chg);   // ends with a barrier
            if (t == 0) {
                const int bits = s_chg;
                p.chg[b] = (uint8_t)bits;
                if (bits) {
                    const int k = b / p.nc;
                    const int c = b - k * p.nc;
                    auto queue = [&](int dep) {
                        if (atomicMax(p.stamp + dep, round + 1) < round + 1)
                            wln[atomicAdd(p.ctl + (cur ^ 1), 1u)] = dep;
                    };
                    if ((bits & kChgLast) && k + 1 < p.nk) queue(b + p.nc);
                    if ((bits & kChgFirst) && c > 0) queue(b - 1);
                    if ((bits & kChgDown) && c + 1 < p.nc) queue(b + 1);
                }
            }
            __syncthreads();   // s_item / s_chg are rewritten by the next take
        }
        if (!grid_barrier(p.ctl + 3, p.ctl + 4, p.err, kLimit)) return;
        // commit: blocks whose output changed now hold it in the other version
        for (unsigned i = blockIdx.x * blockDim.x + t; i < nwork; i += gridDim.x * blockDim.x) {
            const int b = __ldcg(wl + i);
            if (__ldcg(p.chg + b) & kChgAny) p.lat[b] = __ldcg(p.lat + b) == 0 ? 1 : 0;
        }
        if (blockIdx.x == 0 && t == 0) {
            p.ctl[2] = 0;
            p.ctl[cur] = 0;
        }
        if (!grid_barrier(p.ctl + 3, p.ctl + 4, p.err, kLimit)) return;
        if (__ldcg(p.ctl + (cur ^ 1)) == 0) break;
    }
    if (blockIdx.x == 0 && t == 0) p.ctl[5] = (unsigned)(round + 1);
}

// every block takes its rows from the input, and all are queued
__global__ void k_dan_blocks_init(DanBlk p)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < p.nblocks; b += gridDim.x * blockDim.x) {
        p.lat[b] = 2;
        p.chg[b] = 0;
        p.stamp[b] = 0;
        p.wl[0][b] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        p.ctl[0] = (unsigned)p.nblocks;
        for (int i = 1; i < 8; i++) p.ctl[i] = 0;
    }
}

// the converged outputs back into the caller's array
template <class Cell>
__global__ void k_dan_blocks_store(DanBlk p, typename CellIO<Cell>::P* __restrict__ dl)
{
    using IO = CellIO<Cell>;
    using P = typename IO::P;
    const long long plane = (long long)p.w * p.h, cells = plane * p.d;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
         i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        const int y = (int)((i - z * plane) / p.w);
        const int pos = (z - p.zfirst) * p.dir;
        if (pos < 0 || pos >= p.nchain) continue;   // the fixed slice
        const int v = p.lat[(pos / p.Z) * p.nc + y / p.R];
        if (v != 2) {
            const P* src = static_cast<const P*>(p.V[v]);
#pragma unroll
            for (int k = 0; k < IO::kWords; k++) dl[IO::kWords * i + k] = src[IO::kWords * i + k];
        }
    }
}

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

int dan_blocks_rows(int dim, int w, int h, int d)
{
    const int tv = tune_get(kTuneDanRows, w);
    if (tv > 0) return tv;
    // small images: the serial engine's launch is cheaper than the rounds
    const long long cells = (long long)w * h * (dim == 3 ? d : 1);
    if (cells < 65536 || w > 8 * kBlkThreads) return kDanSerial;
    return 8;
}

size_t dan_blocks_workspace_bytes(int dim, int w, int h, int d, int R)
{
    const size_t cb = dim == 3 ? 6 : 4;
    const size_t cells = (size_t)w * h * (dim == 3 ? d : 1);
    const int nc = (h + R - 1) / R;
    const size_t nb = (size_t)nc * (dim == 3 ? d : 1);
    return 2 * al256(cells * cb) + 2 * al256(nb * w * cb) + 2 * al256(nb) + 3 * al256(nb * sizeof(int)) + 256;
}

template <class Cell, int kDim, int S, int T>
static bool run_phase(DanBlk& p, void* dl, cudaStream_t st)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dan_blocks<Cell, kDim, S, T>, T, 0) !=
            cudaSuccess ||
        per_sm < 1)
        return false;
    const int resident = per_sm * g_num_sms;
    // slices per block: long enough that few rounds are needed, short enough
    // that about four block columns per resident CTA keep every SM busy, and
    // at most 16 (on 1024^3 noise, 16 slices ran 686 -> 553 ms against the
    // 110 the column rule gives; 32 and 64 were slower than 16)
    int Z = tune_get(kTuneDanSlices, p.w);
    if (Z < 1) {
        const long long cols = 4LL * resident;
        Z = (int)((long long)p.nchain * p.nc / cols);
        if (Z < 1) Z = 1;
        if (Z > 16) Z = 16;
    }
    if (Z > p.nchain) Z = p.nchain;
    p.Z = Z;
    p.nk = (p.nchain + Z - 1) / Z;
    p.nblocks = p.nk * p.nc;
    p.max_rounds = 2 * p.nblocks + 8;
    k_dan_blocks_init<<<(p.nblocks + 255) / 256, 256, 0, st>>>(p);
    int grid = resident < p.nblocks ? resident : p.nblocks;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(T);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_dan_blocks<Cell, kDim, S, T>, p) != cudaSuccess) return false;
    const long long cells = (long long)p.w * p.h * p.d;
    long long gb = (cells + 255) / 256;
    if (gb > (long long)g_num_sms * 32) gb = (long long)g_num_sms * 32;
    k_dan_blocks_store<Cell><<<(int)gb, 256, 0, st>>>(p, static_cast<typename CellIO<Cell>::P*>(dl));
    return true;
}

template <class Cell, int kDim, int S, int T>
static bool run_all(int w, int h, int d, int cw, int R, void* deltas, void* ws, int* err, cudaStream_t st)
{
    const size_t cb = kDim == 3 ? 6 : 4;
    const size_t cells = (size_t)w * h * d;
    const int nc = (h + R - 1) / R;
    const int nb = nc * d;   // (slice, chunk) pairs: down-boundary row slots, and a bound on the blocks
    char* q = static_cast<char*>(ws);
    DanBlk p{};
    p.A = deltas;
    p.V[0] = q;
    q += al256(cells * cb);
    p.V[1] = q;
    q += al256(cells * cb);
    p.DB[0] = q;
    q += al256((size_t)nb * w * cb);
    p.DB[1] = q;
    q += al256((size_t)nb * w * cb);
    p.lat = reinterpret_cast<uint8_t*>(q);
    q += al256(nb);
    p.chg = reinterpret_cast<uint8_t*>(q);
    q += al256(nb);
    p.stamp = reinterpret_cast<int*>(q);
    q += al256((size_t)nb * sizeof(int));
    p.wl[0] = reinterpret_cast<int*>(q);
    q += al256((size_t)nb * sizeof(int));
    p.wl[1] = reinterpret_cast<int*>(q);
    q += al256((size_t)nb * sizeof(int));
    p.ctl = reinterpret_cast<unsigned*>(q);
    p.err = err;
    p.w = w;
    p.h = h;
    p.d = d;
    p.R = R;
    p.nc = nc;
    p.cw = cw;
    if (kDim == 2) {
        p.dir = 1;
        p.zfirst = 0;
        p.nchain = 1;
        return run_phase<Cell, kDim, S, T>(p, deltas, st);
    }
    // slices 1..d-1 pull from the slice before, then d-2..0 from the slice after
    p.dir = 1;
    p.zfirst = 1;
    p.nchain = d - 1;
    if (!run_phase<Cell, kDim, S, T>(p, deltas, st)) return false;
    p.dir = -1;
    p.zfirst = d - 2;
    return run_phase<Cell, kDim, S, T>(p, deltas, st);
}

size_t danielsson_workspace_bytes(int dim, int w, int h, int d)
{
    const int R = dan_blocks_rows(dim, w, h, d);
    if (R >= kDanSerial || w > 8 * kBlkThreads) return 0;
    return dan_blocks_workspace_bytes(dim, w, h, d, R);
}

bool run_danielsson(int dim, void* deltas, int w, int h, int d, int cw, void* ws, size_t ws_bytes, int* err,
                    cudaStream_t st)
{
    const int R = dan_blocks_rows(dim, w, h, d);
    if (ws && R < kDanSerial && ws_bytes >= dan_blocks_workspace_bytes(dim, w, h, d, R) &&
        launch_danielsson_blocks(dim, deltas, w, h, d, cw, R, ws, err, st))
        return true;
    launch_danielsson(dim, deltas, w, h, d, cw, st);
    return false;
}

bool launch_danielsson_blocks(int dim, void* deltas, int w, int h, int d, int cw, int R, void* ws, int* err,
                              cudaStream_t st)
{
    if (dim == 3 && d < 2) return true;   // the reference's slice loops do not run
    ProfScope ps("danielsson_blocks", st);
    // cells per thread: tuned, else the fewest that keep the row within 128
    // threads in 3D (short segments, CTAs of 2-4 warps, many blocks per SM;
    // cells stop at 4 per thread, where the register file still holds every
    // array) and within 256 in 2D, where an image has fewer blocks than the
    // GPU has SMs and the widest CTA finishes a block soonest (1024^2, 100
    // points: 1.96 ms at 128 threads, 1.37 ms at 256)
    int s = tune_get(dim == 2 ? kTuneDan2 : kTuneDan3, w);
    if (s != 1 && s != 2 && s != 4 && s != 8) {
        const int tmax = dim == 2 ? kBlkThreads : 128;
        s = 1;
        while ((w + s - 1) / s > tmax && s < (dim == 3 ? 4 : 8)) s *= 2;
    }
    while ((w + s - 1) / s > kBlkThreads && s < 8) s *= 2;
    const int nseg = (w + s - 1) / s;
    if (nseg > kBlkThreads) return false;
    const int t = nseg <= 64 ? 64 : (nseg <= 128 ? 128 : 256);
#define DOL_BLK_RUN(SV, TV)                                                                             \
    return dim == 2 ? run_all<C2, 2, SV, TV>(w, h, 1, cw, R, deltas, ws, err, st)                     \
                    : run_all<C3, 3, SV, TV>(w, h, d, cw, R, deltas, ws, err, st);
#define DOL_BLK_CASE(SV)                                                                                \
    case SV:                                                                                            \
        if (t == 64) { DOL_BLK_RUN(SV, 64) }                                                            \
        if (t == 128) { DOL_BLK_RUN(SV, 128) }                                                          \
        DOL_BLK_RUN(SV, 256)
    switch (s) {
        DOL_BLK_CASE(1)
        DOL_BLK_CASE(2)
        DOL_BLK_CASE(4)
        DOL_BLK_CASE(8)
        default: break;
    }
#undef DOL_BLK_CASE
#undef DOL_BLK_RUN
    return false;
}

}  // namespace dolk
