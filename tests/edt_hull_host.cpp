// Host build of the EDT's lower-envelope routines (csrc/hull.cuh) for the CPU
// tests: the same __host__ __device__ code the line kernel runs, driven here
// one tile at a time (segment hulls, the merge tree, the per-cell walk).
#include <vector>

#include "hull.cuh"

template <typename TIn, int SB>
static void run_tile(int n, int TX, const TIn* F0, const TIn* F1, uint32_t* best, uint8_t* none)
{
    const int nseg = (n + SB - 1) / SB;
    std::vector<uint32_t> HM(2 * (size_t)TX * nseg);
    for (int seg = 0; seg < nseg; seg++)
        for (int col = 0; col < TX; col++) dolk::hull_build<TIn, SB>(F0, F1, HM.data(), TX, nseg, n, col, seg);
    for (int half = 1; half < nseg; half <<= 1)
        for (int lo = 0; lo + half < nseg; lo += 2 * half) {
            const int mid = lo + half, hi = mid + half < nseg ? mid + half : nseg;
            for (int sc = 0; sc < 2 * TX; sc++)
                dolk::hull_merge<TIn, SB>(sc >= TX ? F1 : F0, HM.data() + (size_t)sc * nseg, TX, sc % TX, lo, mid, hi);
        }
    for (int seg = 0; seg < nseg; seg++)
        for (int col = 0; col < TX; col++)
            dolk::hull_query<TIn, SB>(F0, F1, HM.data(), TX, nseg, n, col, seg, [&](int p, int, uint32_t b, bool nn) {
                best[(size_t)p * TX + col] = b;
                none[(size_t)p * TX + col] = nn ? 1 : 0;
            });
}

// F0 / F1: split tiles of (32 * ceil(n / 32)) rows x TX columns, position 0 first
// sb: cells per segment, 32 or 16 (the kernel's 8-column tiles)
extern "C" void hull_tile_u16(int n, int TX, const uint16_t* F0, const uint16_t* F1, uint32_t* best, uint8_t* none,
                              int sb)
{
    if (sb == 16)
        run_tile<uint16_t, 16>(n, TX, F0, F1, best, none);
    else
        run_tile<uint16_t, 32>(n, TX, F0, F1, best, none);
}

extern "C" void hull_tile_u32(int n, int TX, const uint32_t* F0, const uint32_t* F1, uint32_t* best, uint8_t* none,
                              int sb)
{
    if (sb == 16)
        run_tile<uint32_t, 16>(n, TX, F0, F1, best, none);
    else
        run_tile<uint32_t, 32>(n, TX, F0, F1, best, none);
}
