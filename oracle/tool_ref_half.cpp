/*
 * tool_ref_half.cpp -- the part of the reference library that the B200
 * library does not replace, for linking the reference's own tool
 * (DistanceOcclusionTool.cpp, compiled unmodified) against libdol_b200.so.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/Makefile, target `tool`).  The reference
 * library is one file; every function the B200 C++ interface
 * (distance-occlusion_b200/shim/DistanceOcclusionB200.h) provides is renamed
 * here by the preprocessor before the file is included as it lies, so this
 * translation unit defines only the rest -- BruteForce, the shadow sweep,
 * InitOccFromBitMask, the Encode* helpers -- under their own names, and its copies
 * of the distance functions under names nothing calls.  The tool's calls of
 * DOL::Danielsson, DOL::InitBorderDeltasFromBitMask, ... then resolve to the
 * GPU library at link time; `nm` on the linked tool shows them undefined.
 */
#define MaskSize                    MaskSize_RefHost
#define CreateBitMask               CreateBitMask_RefHost
#define DestroyBitMask              DestroyBitMask_RefHost
#define BitMaskAddPoints            BitMaskAddPoints_RefHost
#define BitMaskAddBlock             BitMaskAddBlock_RefHost
#define InitDistancesFromBitMask    InitDistancesFromBitMask_RefHost
#define Chamfer                     Chamfer_RefHost
#define Felzenszwalb                Felzenszwalb_RefHost
#define InitDeltasFromBitMask       InitDeltasFromBitMask_RefHost
#define InitBorderDeltasFromBitMask InitBorderDeltasFromBitMask_RefHost
#define FastSweep                   FastSweep_RefHost
#define Danielsson                  Danielsson_RefHost
#define JumpFlood                   JumpFlood_RefHost
#define InitDirWFromBitMask         InitDirWFromBitMask_RefHost
#define OcclusionSweep              OcclusionSweep_RefHost

#include "DistanceOcclusionLib.cpp"
