/*
 * ref_wrap.cpp -- C entry points into the UNMODIFIED reference library.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file
 * with -I pointing at the reference checkout, so the translation unit below
 * includes DistanceOcclusionLib.cpp exactly as it lies there (built with the
 * reference's own -O3, no OpenMP, as its Makefile does).  Including the .cpp
 * rather than linking it gives access to the file-local 1D Felzenszwalb
 * routine (DistanceOcclusionLib.cpp:1026-1062), which the 3D restatement below
 * applies along z, y and x -- the reference has no 3D Felzenszwalb.
 *
 * The output, oracle/_ref/libdolref.so, is git-ignored and never shipped; it
 * pins the C restatement in dol_oracle.c and serves as the timed CPU
 * baseline ("kind": "reference").
 */
#include "DistanceOcclusionLib.cpp"

#include <thread>
#include <vector>

extern "C" {

void ref_add_points_2d(int w, int h, int n, uint32_t seed, uint32_t* mask) { DOL::BitMaskAddPoints(w, h, n, seed, mask); }
void ref_add_points_3d(int w, int h, int d, int n, uint32_t seed, uint32_t* mask) { DOL::BitMaskAddPoints(w, h, d, n, seed, mask); }
void ref_add_block_2d(int w, int h, int sides, uint32_t* mask) { DOL::BitMaskAddBlock(w, h, sides, mask); }
void ref_add_block_3d(int w, int h, int d, int sides, uint32_t* mask) { DOL::BitMaskAddBlock(w, h, d, sides, mask); }

void ref_init_distances_2d(int w, int h, const uint32_t* mask, float* dist) { DOL::InitDistancesFromBitMask(w, h, mask, dist); }
void ref_init_deltas_2d(int w, int h, const uint32_t* mask, DOL::cCellDelta2* dl, int invert) { DOL::InitDeltasFromBitMask(w, h, mask, dl, invert != 0); }
void ref_init_deltas_3d(int w, int h, int d, const uint32_t* mask, DOL::cCellDelta3* dl, int invert) { DOL::InitDeltasFromBitMask(w, h, d, mask, dl, invert != 0); }
void ref_border_init_2d(int w, int h, const uint32_t* mask, DOL::cCellDelta2* dl) { DOL::InitBorderDeltasFromBitMask(w, h, mask, dl); }
void ref_border_init_3d(int w, int h, int d, const uint32_t* mask, DOL::cCellDelta3* dl) { DOL::InitBorderDeltasFromBitMask(w, h, d, mask, dl); }

void ref_danielsson_2d(int w, int h, DOL::cCellDelta2* dl, int cw) { DOL::Danielsson(w, h, dl, cw); }
void ref_danielsson_3d(int w, int h, int d, DOL::cCellDelta3* dl, int cw) { DOL::Danielsson(w, h, d, dl, cw); }
void ref_fastsweep_2d(int w, int h, DOL::cCellDelta2* dl, int cw) { DOL::FastSweep(w, h, dl, cw); }
void ref_fastsweep_3d(int w, int h, int d, DOL::cCellDelta3* dl, int cw) { DOL::FastSweep(w, h, d, dl, cw); }
void ref_jumpflood_2d(int w, int h, DOL::cCellDelta2* dl, int cw) { DOL::JumpFlood(w, h, dl, cw); }
void ref_jumpflood_3d(int w, int h, int d, DOL::cCellDelta3* dl, int cw) { DOL::JumpFlood(w, h, d, dl, cw); }
void ref_bruteforce_2d(int w, int h, DOL::cCellDelta2* dl, int cw) { DOL::BruteForce(w, h, dl, cw); }
void ref_bruteforce_3d(int w, int h, int d, DOL::cCellDelta3* dl, int cw) { DOL::BruteForce(w, h, d, dl, cw); }
void ref_felzenszwalb_2d(int w, int h, float* dist) { DOL::Felzenszwalb(w, h, dist); }
void ref_init_distances_2d_i16(int w, int h, const uint32_t* mask, int16_t* dist, int16_t max_d) { DOL::InitDistancesFromBitMask(w, h, mask, dist, max_d); }
void ref_init_distances_2d_i32(int w, int h, const uint32_t* mask, int32_t* dist, int32_t max_d) { DOL::InitDistancesFromBitMask(w, h, mask, dist, max_d); }
int ref_chamfer_2d_i16(int w, int h, int16_t* dist) { return DOL::Chamfer(w, h, dist); }
int ref_chamfer_2d_i32(int w, int h, int32_t* dist) { return DOL::Chamfer(w, h, dist); }
void ref_init_dirw_2d(int w, int h, const uint32_t* mask, float* dirW) { DOL::InitDirWFromBitMask(w, h, mask, dirW); }
void ref_init_dirw_3d(int w, int h, int d, const uint32_t* mask, float* dirW) { DOL::InitDirWFromBitMask(w, h, d, mask, dirW); }
void ref_occlusion_sweep_2d(int w, int h, float* dirW) { DOL::OcclusionSweep(w, h, dirW); }
void ref_occlusion_sweep_3d(int w, int h, int d, float* dirW) { DOL::OcclusionSweep(w, h, d, dirW); }
void ref_occlusion_sweep_3d_io(int w, int h, int d, const float* in, float* out) { DOL::OcclusionSweep(w, h, d, in, out); }

/* 3D restatement on the reference's own 1D routine: z, then y, then x.  Lines
 * are split over `threads` host threads, each with private v/z/line scratch
 * (the reference's OpenMP pragmas share that scratch, so they are not used). */
void ref_felzenszwalb_3d(int w, int h, int d, float* dist, int threads)
{
    if (threads < 1) threads = 1;
    const size_t ss = (size_t)w * h;
    const int nmax = (w > h ? (w > d ? w : d) : (h > d ? h : d));

    auto run = [&](int pass, int t) {
        std::vector<int> v(nmax);
        std::vector<float> z(nmax + 1), line(nmax);
        if (pass == 0) {            /* along z: lines indexed by (y, x) */
            for (size_t c = t; c < ss; c += threads) {
                float* col = dist + c;
                ::Felzenszwalb(d, (int)ss, col, line.data(), v.data(), z.data());
                for (int q = 0; q < d; q++) col[(size_t)q * ss] = line[q];
            }
        } else if (pass == 1) {     /* along y: lines indexed by (z, x) */
            for (size_t c = t; c < (size_t)d * w; c += threads) {
                size_t k = c / w, x = c % w;
                float* col = dist + k * ss + x;
                ::Felzenszwalb(h, w, col, line.data(), v.data(), z.data());
                for (int q = 0; q < h; q++) col[(size_t)q * w] = line[q];
            }
        } else {                    /* along x: lines indexed by (z, y) */
            for (size_t c = t; c < (size_t)d * h; c += threads) {
                float* row = dist + c * w;
                ::Felzenszwalb(w, 1, row, line.data(), v.data(), z.data());
                for (int q = 0; q < w; q++) row[q] = line[q];
            }
        }
    };
    for (int pass = 0; pass < 3; pass++) {
        if (threads == 1) { run(pass, 0); continue; }
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++) pool.emplace_back(run, pass, t);
        for (auto& th : pool) th.join();
    }
}

/* One pass of the same 3D restatement over a rectangle of its lines, for
 * timing bounded samples of a large volume.  pass 0: z lines (a = y, b = x);
 * 1: y lines (a = z, b = x); 2: x rows (a = z, b = y); lines (a, b) with
 * a0 <= a < a1, b0 <= b < b1.  Reads src, writes dst (both whole w*h*d
 * volumes, so strides are those of the full volume; dst may be src: every
 * line goes through a private buffer).  Each of `threads` host threads takes
 * one contiguous block of the lines in (a, b) order, as a static loop
 * schedule would. */
void ref_felzenszwalb_3d_pass(int w, int h, int d, const float* src, float* dst, int pass, int a0, int a1, int b0,
                              int b1, int threads)
{
    if (threads < 1) threads = 1;
    const size_t ss = (size_t)w * h;
    const int n = pass == 0 ? d : (pass == 1 ? h : w);
    const size_t stride = pass == 0 ? ss : (pass == 1 ? (size_t)w : 1);
    const long long nb = b1 - b0, lines = (long long)(a1 - a0) * nb;
    auto line_base = [&](long long i) -> size_t {
        const size_t a = (size_t)(a0 + i / nb), b = (size_t)(b0 + i % nb);
        if (pass == 0) return a * w + b;         /* (y, x): column through all slices */
        if (pass == 1) return a * ss + b;        /* (z, x): column of slice z */
        return a * ss + b * w;                   /* (z, y): row */
    };
    auto run = [&](int t) {
        std::vector<int> v(n);
        std::vector<float> z(n + 1), line(n);
        const long long lo = lines * t / threads, hi = lines * (t + 1) / threads;
        for (long long i = lo; i < hi; i++) {
            const size_t base = line_base(i);
            ::Felzenszwalb(n, (int)stride, src + base, line.data(), v.data(), z.data());
            float* o = dst + base;
            for (int q = 0; q < n; q++) o[(size_t)q * stride] = line[q];
        }
    };
    if (threads == 1) { run(0); return; }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(run, t);
    for (auto& th : pool) th.join();
}

/* The signed field from the two squared transforms, as the tool's two-pass
 * path forms it (DistanceOcclusionTool.cpp:54-61, :1036): out = sqrtf(occ) -
 * sqrtf(emp), over n floats split across `threads` host threads. */
void ref_sqrt_diff(long long n, const float* occ, const float* emp, float* out, int threads)
{
    if (threads < 1) threads = 1;
    auto run = [&](int t) {
        const long long lo = n * t / threads, hi = n * (t + 1) / threads;
        for (long long i = lo; i < hi; i++) out[i] = sqrtf(occ[i]) - sqrtf(emp[i]);
    };
    if (threads == 1) { run(0); return; }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(run, t);
    for (auto& th : pool) th.join();
}

}  /* extern "C" */
