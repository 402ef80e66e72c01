// DistanceOcclusionB200.cpp -- namespace DOL over the C ABI (see the header).
// Built into libdol_b200.so by build.py.
#include "DistanceOcclusionB200.h"

#include <cuda_runtime.h>
#include <string.h>

#include "dol_b200.h"

#pragma GCC visibility push(default)

namespace
{
    void Check(dol_status s)
    {
        if (s != DOL_OK) throw DOL::Error((int)s, std::string("dol_b200: ") + dol_last_error());
    }

    void CheckCuda(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess) throw DOL::Error(DOL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }

    // A device buffer that lives for one call.
    struct Dev
    {
        void* p = nullptr;
        explicit Dev(size_t bytes) { if (bytes) CheckCuda(cudaMalloc(&p, bytes), "cudaMalloc"); }
        ~Dev() { if (p) cudaFree(p); }
        Dev(const Dev&) = delete;
        Dev& operator=(const Dev&) = delete;
        template <class T> T* as() const { return static_cast<T*>(p); }
        void up(const void* h, size_t n) { CheckCuda(cudaMemcpy(p, h, n, cudaMemcpyHostToDevice), "copy to device"); }
        void down(void* h, size_t n) const { CheckCuda(cudaMemcpy(h, p, n, cudaMemcpyDeviceToHost), "copy to host"); }
    };

    size_t MaskBytes(int w, int h, int d) { return dol_mask_words(w, h, d) * sizeof(uint32_t); }

    void Finish() { Check(dol_sync(nullptr)); }

    template <class Cell, class Fn>
    void InPlace(Cell* host, size_t cells, Fn&& run)
    {
        Dev dl(cells * sizeof(Cell));
        dl.up(host, cells * sizeof(Cell));
        run(dl.as<Cell>());
        Finish();
        dl.down(host, cells * sizeof(Cell));
    }
}

namespace DOL
{
    int MaskSize(int w) { return (w + 31) / 32; }
    int MaskSize(int w, int h) { return ((w + 31) / 32) * h; }
    int MaskSize(int w, int h, int d) { return ((w + 31) / 32) * h * d; }

    uint32_t* CreateBitMask(int w, int h)
    {
        size_t n = (size_t)MaskSize(w, h);
        uint32_t* m = new uint32_t[n];
        memset(m, 0, n * sizeof(uint32_t));
        return m;
    }

    uint32_t* CreateBitMask(int w, int h, int d)
    {
        size_t n = (size_t)MaskSize(w, h, d);
        uint32_t* m = new uint32_t[n];
        memset(m, 0, n * sizeof(uint32_t));
        return m;
    }

    void DestroyBitMask(uint32_t*& mask)
    {
        delete[] mask;
        mask = nullptr;
    }

    void BitMaskAddPoints(int w, int h, int n, uint32_t seed, uint32_t mask[]) { dol_add_points_2d(w, h, n, seed, mask); }
    void BitMaskAddPoints(int w, int h, int d, int n, uint32_t seed, uint32_t mask[]) { dol_add_points_3d(w, h, d, n, seed, mask); }
    void BitMaskAddBlock(int w, int h, int sides, uint32_t mask[]) { dol_add_block_2d(w, h, sides, mask); }
    void BitMaskAddBlock(int w, int h, int d, int sides, uint32_t mask[]) { dol_add_block_3d(w, h, d, sides, mask); }

    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], float distances[], float maxD)
    {
        Dev dm(MaskBytes(w, h, 1)), df((size_t)w * h * sizeof(float));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_distances_2d(w, h, dm.as<uint32_t>(), df.as<float>(), maxD, nullptr));
        Finish();
        df.down(distances, (size_t)w * h * sizeof(float));
    }

    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], int16_t distances[], int16_t maxD)
    {
        Dev dm(MaskBytes(w, h, 1)), df((size_t)w * h * sizeof(int16_t));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_distances_2d_i16(w, h, dm.as<uint32_t>(), df.as<int16_t>(), maxD, nullptr));
        Finish();
        df.down(distances, (size_t)w * h * sizeof(int16_t));
    }

    void InitDistancesFromBitMask(int w, int h, const uint32_t mask[], int32_t distances[], int32_t maxD)
    {
        Dev dm(MaskBytes(w, h, 1)), df((size_t)w * h * sizeof(int32_t));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_distances_2d_i32(w, h, dm.as<uint32_t>(), df.as<int32_t>(), maxD, nullptr));
        Finish();
        df.down(distances, (size_t)w * h * sizeof(int32_t));
    }

    int Chamfer(int w, int h, int16_t distances[])
    {
        int m = 3;
        InPlace(distances, (size_t)w * h, [&](int16_t* d) { Check(dol_chamfer_2d_i16(w, h, d, &m, nullptr)); });
        return m;
    }

    int Chamfer(int w, int h, int32_t distances[])
    {
        int m = 3;
        InPlace(distances, (size_t)w * h, [&](int32_t* d) { Check(dol_chamfer_2d_i32(w, h, d, &m, nullptr)); });
        return m;
    }

    void Felzenszwalb(int w, int h, float distances[])
    {
        InPlace(distances, (size_t)w * h, [&](float* d) { Check(dol_felzenszwalb_2d(w, h, d, nullptr, 0, nullptr)); });
    }

    // --- occlusion -----------------------------------------------------------------
    void InitDirWFromBitMask(int w, int h, const uint32_t mask[], float dirW4[])
    {
        const size_t n = 4 * (size_t)w * h * sizeof(float);
        Dev dm(MaskBytes(w, h, 1)), dd(n);
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_dirw_2d(w, h, dm.as<uint32_t>(), dd.as<float>(), nullptr));
        Finish();
        dd.down(dirW4, n);
    }

    void InitDirWFromBitMask(int w, int h, int d, const uint32_t mask[], float dirW8[])
    {
        const size_t n = 8 * (size_t)w * h * d * sizeof(float);
        Dev dm(MaskBytes(w, h, d)), dd(n);
        dm.up(mask, MaskBytes(w, h, d));
        Check(dol_init_dirw_3d(w, h, d, dm.as<uint32_t>(), dd.as<float>(), nullptr));
        Finish();
        dd.down(dirW8, n);
    }

    void OcclusionSweep(int w, int h, float dirW4[])
    {
        InPlace(dirW4, 4 * (size_t)w * h, [&](float* p) { Check(dol_occlusion_sweep_2d(w, h, p, nullptr)); });
    }

    void OcclusionSweep(int w, int h, int d, float dirW8[])
    {
        InPlace(dirW8, 8 * (size_t)w * h * d, [&](float* p) { Check(dol_occlusion_sweep_3d(w, h, d, p, nullptr)); });
    }

    void OcclusionSweep(int w, int h, int d, const float inDirW8[], float outDirW8[])
    {
        // out goes up too: the reference leaves each plane's starting cell as it was
        const size_t n = 8 * (size_t)w * h * d * sizeof(float);
        Dev di(n), dout(n);
        di.up(inDirW8, n);
        dout.up(outDirW8, n);
        Check(dol_occlusion_sweep_3d_io(w, h, d, di.as<float>(), dout.as<float>(), nullptr));
        Finish();
        dout.down(outDirW8, n);
    }

    void InitDeltasFromBitMask(int w, int h, const uint32_t mask[], cCellDelta2 delta[], bool invert)
    {
        Dev dm(MaskBytes(w, h, 1)), dd((size_t)w * h * sizeof(cCellDelta2));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_deltas_2d(w, h, dm.as<uint32_t>(), dd.as<dol_delta2>(), invert ? 1 : 0, nullptr));
        Finish();
        dd.down(delta, (size_t)w * h * sizeof(cCellDelta2));
    }

    void InitDeltasFromBitMask(int w, int h, int d, const uint32_t mask[], cCellDelta3 delta[], bool invert)
    {
        size_t cells = (size_t)w * h * d;
        Dev dm(MaskBytes(w, h, d)), dd(cells * sizeof(cCellDelta3));
        dm.up(mask, MaskBytes(w, h, d));
        Check(dol_init_deltas_3d(w, h, d, dm.as<uint32_t>(), dd.as<dol_delta3>(), invert ? 1 : 0, nullptr));
        Finish();
        dd.down(delta, cells * sizeof(cCellDelta3));
    }

    void InitBorderDeltasFromBitMask(int w, int h, const uint32_t mask[], cCellDelta2 delta[])
    {
        Dev dm(MaskBytes(w, h, 1)), dd((size_t)w * h * sizeof(cCellDelta2));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_init_border_2d(w, h, dm.as<uint32_t>(), dd.as<dol_delta2>(), nullptr));
        Finish();
        dd.down(delta, (size_t)w * h * sizeof(cCellDelta2));
    }

    void InitBorderDeltasFromBitMask(int w, int h, int d, const uint32_t mask[], cCellDelta3 delta[])
    {
        size_t cells = (size_t)w * h * d;
        Dev dm(MaskBytes(w, h, d)), dd(cells * sizeof(cCellDelta3));
        dm.up(mask, MaskBytes(w, h, d));
        Check(dol_init_border_3d(w, h, d, dm.as<uint32_t>(), dd.as<dol_delta3>(), nullptr));
        Finish();
        dd.down(delta, cells * sizeof(cCellDelta3));
    }

    void FastSweep(int w, int h, cCellDelta2 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h, [&](cCellDelta2* d) {
            Check(dol_fastsweep_2d(w, h, reinterpret_cast<dol_delta2*>(d), cw, nullptr));
        });
    }

    void FastSweep(int w, int h, int d, cCellDelta3 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h * d, [&](cCellDelta3* p) {
            Check(dol_fastsweep_3d(w, h, d, reinterpret_cast<dol_delta3*>(p), cw, nullptr, 0, nullptr));
        });
    }

    void Danielsson(int w, int h, cCellDelta2 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h, [&](cCellDelta2* d) {
            Check(dol_danielsson_2d(w, h, reinterpret_cast<dol_delta2*>(d), cw, nullptr));
        });
    }

    void Danielsson(int w, int h, int d, cCellDelta3 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h * d, [&](cCellDelta3* p) {
            Check(dol_danielsson_3d(w, h, d, reinterpret_cast<dol_delta3*>(p), cw, nullptr));
        });
    }

    void JumpFlood(int w, int h, cCellDelta2 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h, [&](cCellDelta2* d) {
            Check(dol_jumpflood_2d(w, h, reinterpret_cast<dol_delta2*>(d), cw, nullptr, 0, nullptr));
        });
    }

    void JumpFlood(int w, int h, int d, cCellDelta3 delta[], int cw)
    {
        InPlace(delta, (size_t)w * h * d, [&](cCellDelta3* p) {
            Check(dol_jumpflood_3d(w, h, d, reinterpret_cast<dol_delta3*>(p), cw, nullptr, 0, nullptr));
        });
    }

    void DistancesFromBitMask(int w, int h, const uint32_t mask[], float out[], int form)
    {
        Dev dm(MaskBytes(w, h, 1)), df((size_t)w * h * sizeof(float));
        dm.up(mask, MaskBytes(w, h, 1));
        Check(dol_edt_mask_2d(w, h, dm.as<uint32_t>(), df.as<float>(), form, nullptr, 0, nullptr));
        Finish();
        df.down(out, (size_t)w * h * sizeof(float));
    }

    void DistancesFromBitMask(int w, int h, int d, const uint32_t mask[], float out[], int form)
    {
        Check(dol_edt_mask_3d_host(w, h, d, mask, out, form));
    }

    void DeltasToDistances(int w, int h, const cCellDelta2 delta[], int cw, const uint32_t signMask[], float out[])
    {
        size_t cells = (size_t)w * h;
        Dev dd(cells * sizeof(cCellDelta2)), df(cells * sizeof(float)), dm(signMask ? MaskBytes(w, h, 1) : 0);
        dd.up(delta, cells * sizeof(cCellDelta2));
        if (signMask) dm.up(signMask, MaskBytes(w, h, 1));
        Check(dol_deltas_to_dist_2d(w, h, dd.as<dol_delta2>(), cw, signMask ? dm.as<uint32_t>() : nullptr,
                                    df.as<float>(), nullptr));
        Finish();
        df.down(out, cells * sizeof(float));
    }

    void DeltasToDistances(int w, int h, int d, const cCellDelta3 delta[], int cw, const uint32_t signMask[], float out[])
    {
        size_t cells = (size_t)w * h * d;
        Dev dd(cells * sizeof(cCellDelta3)), df(cells * sizeof(float)), dm(signMask ? MaskBytes(w, h, d) : 0);
        dd.up(delta, cells * sizeof(cCellDelta3));
        if (signMask) dm.up(signMask, MaskBytes(w, h, d));
        Check(dol_deltas_to_dist_3d(w, h, d, dd.as<dol_delta3>(), cw, signMask ? dm.as<uint32_t>() : nullptr,
                                    df.as<float>(), nullptr));
        Finish();
        df.down(out, cells * sizeof(float));
    }
}

#pragma GCC visibility pop
