// DistanceOcclusionB200.h -- C++ host interface of the B200 distance-field
// library, shaped like the distance-field half of DistanceOcclusionLib.h
// (namespace DOL, same function names, argument order, array layouts and
// in-place semantics), so code written against the reference's distance
// functions compiles against this header and runs them on the GPU.
//
// Arrays are HOST memory, as in the reference; each call copies its inputs to
// the device, runs the CUDA kernels through the C ABI (dol_b200.h) and copies
// the results back.  Callers holding device buffers should call the C ABI
// directly and skip the copies.  Failures throw DOL::Error (the reference has
// no error reporting; it would crash or write out of bounds instead).
//
// Of the reference's occlusion routines, InitDirWFromBitMask and
// OcclusionSweep run here on the GPU; ShadowSweep, InitOccFromBitMask and the
// Encode* helpers stay with the reference library on the host.
#ifndef DISTANCE_OCCLUSION_B200_H
#define DISTANCE_OCCLUSION_B200_H

#include <float.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace DOL
{
    struct Error : std::runtime_error
    {
        int status;
        Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
    };

    // --- bitmasks: rows padded to whole uint32 words, LSB first ---------------
    int MaskSize(int w);
    int MaskSize(int w, int h);
    int MaskSize(int w, int h, int d);

    uint32_t* CreateBitMask (int w, int h);
    uint32_t* CreateBitMask (int w, int h, int d);
    void      DestroyBitMask(uint32_t*& mask);

    void BitMaskAddPoints(int w, int h,        int n, uint32_t seed, uint32_t mask[]);
    void BitMaskAddPoints(int w, int h, int d, int n, uint32_t seed, uint32_t mask[]);
    void BitMaskAddBlock (int w, int h,        int sides, uint32_t mask[]);
    void BitMaskAddBlock (int w, int h, int d, int sides, uint32_t mask[]);

    // --- cell deltas: offset from a cell to its closest boundary point --------
    struct cCellDelta2 { int16_t x; int16_t y; };
    struct cCellDelta3 { int16_t x; int16_t y; int16_t z; };

    const int16_t kMaxDelta2 = INT16_MAX;
    const int16_t kMaxDelta3 = 25000;

    // --- distances -----------------------------------------------------------------
    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], int16_t distances[], int16_t maxD = INT16_MAX);
    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], int32_t distances[], int32_t maxD = INT32_MAX);
    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], float distances[], float maxD = FLT_MAX);
    int  Chamfer(int w, int h, int16_t distances[]);   // returns the multiplier (3)
    int  Chamfer(int w, int h, int32_t distances[]);
    void Felzenszwalb(int w, int h, float distances[]);   // squared distances, in place

    // --- delta methods --------------------------------------------------------------
    void InitDeltasFromBitMask(int w, int h,        const uint32_t mask[], cCellDelta2 delta[], bool invert = false);
    void InitDeltasFromBitMask(int w, int h, int d, const uint32_t mask[], cCellDelta3 delta[], bool invert = false);

    void InitBorderDeltasFromBitMask(int w, int h,        const uint32_t mask[], cCellDelta2 delta[]);
    void InitBorderDeltasFromBitMask(int w, int h, int d, const uint32_t mask[], cCellDelta3 delta[]);

    void FastSweep (int w, int h,        cCellDelta2 delta[], int cw = 1);
    void FastSweep (int w, int h, int d, cCellDelta3 delta[], int cw = 1);
    void Danielsson(int w, int h,        cCellDelta2 delta[], int cw = 1);
    void Danielsson(int w, int h, int d, cCellDelta3 delta[], int cw = 1);
    void JumpFlood (int w, int h,        cCellDelta2 delta[], int cw = 1);
    void JumpFlood (int w, int h, int d, cCellDelta3 delta[], int cw = 1);

    // --- occlusion: direction-weight planes (4 in 2D, 8 in 3D) and their sweeps --------
    void InitDirWFromBitMask(int w, int h,        const uint32_t mask[], float dirW4[]);
    void InitDirWFromBitMask(int w, int h, int d, const uint32_t mask[], float dirW8[]);
    void OcclusionSweep(int w, int h,        float dirW4[]);
    void OcclusionSweep(int w, int h, int d, float dirW8[]);
    void OcclusionSweep(int w, int h, int d, const float inDirW8[], float outDirW8[]);

    // --- additions with no reference counterpart -----------------------------------
    // Exact EDT straight from the mask: form 0 squared, 1 distance, 2 signed
    // (distance to set cells minus distance to clear cells); 2D and 3D.
    void DistancesFromBitMask(int w, int h,        const uint32_t mask[], float out[], int form = 1);
    void DistancesFromBitMask(int w, int h, int d, const uint32_t mask[], float out[], int form = 1);
    // Deltas -> float distances: sqrt(len^2) / cw, negated where signMask (if given) is set.
    void DeltasToDistances(int w, int h,        const cCellDelta2 delta[], int cw, const uint32_t signMask[], float out[]);
    void DeltasToDistances(int w, int h, int d, const cCellDelta3 delta[], int cw, const uint32_t signMask[], float out[]);
}

#endif
