// Exercises the C++ host interface (namespace DOL, shim/DistanceOcclusionB200.h)
// the way the reference's tool drives DistanceOcclusionLib: make a mask, run a
// delta method, write the result.  Usage:
//   shim_driver <method 0|1|2|4> <signed 0|1> <w> <h> <d> <points> <seed> <out.bin>
// d = 0 selects 2D.  The output is the raw delta array (cCellDelta2/3 bytes);
// method 4 (Chamfer, 2D only, as the tool's GenerateDistanceChamfer) writes the
// int16 distances instead.
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "DistanceOcclusionB200.h"

using namespace DOL;

int main(int argc, char** argv)
{
    if (argc < 9) return 2;
    int method = atoi(argv[1]), sgn = atoi(argv[2]), w = atoi(argv[3]), h = atoi(argv[4]), d = atoi(argv[5]);
    int points = atoi(argv[6]);
    uint32_t seed = (uint32_t)atoi(argv[7]);
    FILE* f = fopen(argv[8], "wb");
    if (!f) return 3;
    try {
        if (d == 0 && method == 4) {
            uint32_t* mask = CreateBitMask(w, h);
            BitMaskAddBlock(w, h, 4, mask);
            BitMaskAddPoints(w, h, points, seed, mask);
            std::vector<int16_t> dist((size_t)w * h);
            InitDistancesFromBitMask(w, h, mask, dist.data(), (int16_t)(INT16_MAX - 16));
            if (Chamfer(w, h, dist.data()) != 3) return 4;
            fwrite(dist.data(), sizeof(int16_t), dist.size(), f);
            DestroyBitMask(mask);
        } else if (d == 0) {
            uint32_t* mask = CreateBitMask(w, h);
            BitMaskAddBlock(w, h, 4, mask);
            BitMaskAddPoints(w, h, points, seed, mask);
            std::vector<cCellDelta2> dl((size_t)w * h);
            if (sgn) InitBorderDeltasFromBitMask(w, h, mask, dl.data());
            else InitDeltasFromBitMask(w, h, mask, dl.data());
            int cw = sgn ? 2 : 1;
            if (method == 0) Danielsson(w, h, dl.data(), cw);
            else if (method == 1) FastSweep(w, h, dl.data(), cw);
            else JumpFlood(w, h, dl.data(), cw);
            fwrite(dl.data(), sizeof(cCellDelta2), dl.size(), f);
            DestroyBitMask(mask);
        } else {
            uint32_t* mask = CreateBitMask(w, h, d);
            BitMaskAddBlock(w, h, d, 6, mask);
            BitMaskAddPoints(w, h, d, points, seed, mask);
            std::vector<cCellDelta3> dl((size_t)w * h * d);
            if (sgn) InitBorderDeltasFromBitMask(w, h, d, mask, dl.data());
            else InitDeltasFromBitMask(w, h, d, mask, dl.data());
            int cw = sgn ? 2 : 1;
            if (method == 0) Danielsson(w, h, d, dl.data(), cw);
            else if (method == 1) FastSweep(w, h, d, dl.data(), cw);
            else JumpFlood(w, h, d, dl.data(), cw);
            fwrite(dl.data(), sizeof(cCellDelta3), dl.size(), f);
            DestroyBitMask(mask);
        }
    } catch (const Error& e) {
        fprintf(stderr, "%s\n", e.what());
        fclose(f);
        return 1;
    }
    fclose(f);
    return 0;
}
