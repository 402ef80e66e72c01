// k_init.cu -- byte-mask packing, plain initialisation and signed border
// initialisation (DistanceOcclusionLib.cpp:183-254, :504-619, :1289-1321,
// :1820-2173; DistanceOcclusionTool.cpp:634-670).
//
// All kernels here are warp-per-32-mask-words: a warp loads 32 consecutive
// mask words (one 128-byte line), and writes the cells of those words as one
// contiguous, coalesced run (the words of a row are contiguous in the cell
// array, and rows follow each other, so 32 consecutive words always map to a
// contiguous range of cells even when the last word of a row is partial).
#include "border.cuh"
#include "kernels.h"

namespace dolk {

// number of live cells in global word `wid`, and the index of its first cell
__device__ __forceinline__ void word_cells(long long wid, int w, int ws, long long* first, int* n)
{
    long long row = wid / ws;
    int k = (int)(wid - row * ws);
    *first = row * (long long)w + 32 * k;
    int m = w - 32 * k;
    *n = m < 32 ? m : 32;
}

// ---- byte mask -> bitmask ---------------------------------------------------
// One warp per 32 words: for each word, lane b reads byte 32k+b of the row
// (a coalesced 32-byte load) and a ballot forms the word.
__global__ void k_pack_bytemask(const uint8_t* __restrict__ bytes, uint32_t* __restrict__ mask, int w,
                                long long nwords, int threshold, int less_than)
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
            int k = (int)(wid - row * ws);
            int x = 32 * k + lane;
            bool bit = false;
            if (x < w) {
                int v = bytes[row * (long long)w + x];
                bit = (v >= threshold) != (less_than != 0);
            }
            uint32_t word = __ballot_sync(0xFFFFFFFFu, bit);
            if (lane == q) mine = word;
        }
        if (base + lane < nwords) mask[base + lane] = mine;
    }
}

// ---- plain initialisation -----------------------------------------------------
// InitDistancesFromBitMask(float) / InitDeltasFromBitMask: 0 where (bit ^ invert),
// the max value elsewhere; padding bits beyond w are ignored.
template <int kDim>
__global__ void k_init_deltas(const uint32_t* __restrict__ mask, void* __restrict__ out, int w, long long nwords,
                              uint32_t invert, uint32_t fill_bits)
{
    const int lane = threadIdx.x & 31;
    const int ws = words_per_row(w);
    long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < nwords; base += nwarps * 32) {
        uint32_t mine = base + lane < nwords ? (mask[base + lane] ^ invert) : 0u;
        for (int q = 0; q < 32; q++) {
            long long wid = base + q;
            if (wid >= nwords) break;
            uint32_t word = __shfl_sync(0xFFFFFFFFu, mine, q);
            long long first;
            int n;
            word_cells(wid, w, ws, &first, &n);
            if (lane < n) {
                bool on = (word >> lane) & 1u;
                long long c = first + lane;
                if (kDim == 2) {
                    uint32_t v = on ? 0u : pack2(C2{kMax2, kMax2});
                    static_cast<uint32_t*>(out)[c] = v;
                } else if (kDim == 3) {
                    int16_t v = on ? 0 : (int16_t)kMax3;
                    int16_t* o = static_cast<int16_t*>(out) + 3 * c;
                    o[0] = v;
                    o[1] = v;
                    o[2] = v;
                } else {   // float distances: kDim == 1
                    static_cast<float*>(out)[c] = on ? 0.0f : __uint_as_float(fill_bits);
                }
            }
        }
    }
}

// ---- signed border initialisation ---------------------------------------------
// Lane q computes the bit planes of word base+q (border2_word / border3_word),
// parks them in shared memory, then the warp writes the words' cells one word
// at a time, lane = bit.
template <int kDim>
__global__ void __launch_bounds__(256) k_init_border(const uint32_t* __restrict__ mask, void* __restrict__ out,
                                                     int w, int h, int d, long long nwords)
{
    constexpr int kPlanes = kDim == 2 ? 5 : 7;
    __shared__ uint32_t planes[8][32][kPlanes + 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int ws = words_per_row(w);
    long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < nwords; base += nwarps * 32) {
        long long wid = base + lane;
        if (wid < nwords) {
            long long row = wid / ws;
            int k = (int)(wid - row * ws);
            if (kDim == 2) {
                Planes2 p = border2_word(w, h, mask, (int)row, k);
                uint32_t* s = planes[wib][lane];
                s[0] = p.mx; s[1] = p.xn; s[2] = p.xs; s[3] = p.yn; s[4] = p.ys;
            } else {
                int z = (int)(row / h), y = (int)(row - (long long)z * h);
                Planes3 p = border3_word(w, h, d, mask, z, y, k);
                uint32_t* s = planes[wib][lane];
                s[0] = p.mx; s[1] = p.xn; s[2] = p.xs; s[3] = p.yn; s[4] = p.ys;
                if (kDim == 3) { s[5] = p.zn; s[6] = p.zs; }
            }
        }
        __syncwarp();
        for (int q = 0; q < 32; q++) {
            long long wq = base + q;
            if (wq >= nwords) break;
            long long first;
            int n;
            word_cells(wq, w, ws, &first, &n);
            if (lane < n) {
                const uint32_t* s = planes[wib][q];
                if (kDim == 2) {
                    Planes2 p{s[0], s[1], s[2], s[3], s[4]};
                    static_cast<uint32_t*>(out)[first + lane] = pack2(decode2(p, lane));
                } else {
                    Planes3 p{s[0], s[1], s[2], s[3], s[4], s[5], s[6]};
                    C3 c = decode3(p, lane);
                    int16_t* o = static_cast<int16_t*>(out) + 3 * (first + lane);
                    o[0] = (int16_t)c.x;
                    o[1] = (int16_t)c.y;
                    o[2] = (int16_t)c.z;
                }
            }
        }
        __syncwarp();
    }
}

// ---- launchers -------------------------------------------------------------------

static int grid_for_words(long long nwords, int threads)
{
    long long warps = (nwords + 31) / 32;
    long long blocks = (warps * 32 + threads - 1) / threads;
    long long cap = (long long)g_num_sms * 16;
    if (blocks > cap) blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

void launch_pack_bytemask(const uint8_t* bytes, uint32_t* mask, int w, long long rows, int threshold, int less_than,
                          cudaStream_t st)
{
    long long nwords = (long long)words_per_row(w) * rows;
    k_pack_bytemask<<<grid_for_words(nwords, 256), 256, 0, st>>>(bytes, mask, w, nwords, threshold, less_than);
}

void launch_init_distances(const uint32_t* mask, float* dist, int w, long long rows, float max_d, cudaStream_t st)
{
    long long nwords = (long long)words_per_row(w) * rows;
    k_init_deltas<1><<<grid_for_words(nwords, 256), 256, 0, st>>>(mask, dist, w, nwords, 0u, float_bits(max_d));
}

void launch_init_deltas(int dim, const uint32_t* mask, void* deltas, int w, long long rows, int invert, cudaStream_t st)
{
    long long nwords = (long long)words_per_row(w) * rows;
    uint32_t inv = invert ? 0xFFFFFFFFu : 0u;
    if (dim == 2)
        k_init_deltas<2><<<grid_for_words(nwords, 256), 256, 0, st>>>(mask, deltas, w, nwords, inv, 0u);
    else
        k_init_deltas<3><<<grid_for_words(nwords, 256), 256, 0, st>>>(mask, deltas, w, nwords, inv, 0u);
}

void launch_init_border(int dim, const uint32_t* mask, void* deltas, int w, int h, int d, cudaStream_t st)
{
    long long nwords = (long long)words_per_row(w) * h * (dim == 3 ? d : 1);
    ProfScope ps("init_border", st);
    if (dim == 2)
        k_init_border<2><<<grid_for_words(nwords, 256), 256, 0, st>>>(mask, deltas, w, h, 1, nwords);
    else
        k_init_border<3><<<grid_for_words(nwords, 256), 256, 0, st>>>(mask, deltas, w, h, d, nwords);
}

}  // namespace dolk
