// MeshSupportB200.cpp -- MSL::CreateBitMaskFromTriangles over the C ABI (see
// the header).  Built into libdol_b200.so by build.py.
#include "MeshSupportB200.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "DistanceOcclusionB200.h"
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

    struct Dev
    {
        void* p = nullptr;
        explicit Dev(size_t bytes) { if (bytes) CheckCuda(cudaMalloc(&p, bytes), "cudaMalloc"); }
        ~Dev() { if (p) cudaFree(p); }
        Dev(const Dev&) = delete;
        Dev& operator=(const Dev&) = delete;
    };
}

namespace MSL
{
    void CreateBitMaskFromTriangles(int triCount, const int indices[], const Vec3f vertices[], const Bounds3f& bbox,
                                    int w, int h, int d, uint32_t mask[])
    {
        // the vertices the triangles use: up to the largest index (or 3 per triangle)
        size_t nv = 0;
        if (indices) {
            for (int i = 0; i < 3 * triCount; i++)
                if ((size_t)indices[i] + 1 > nv) nv = (size_t)indices[i] + 1;
        } else {
            nv = 3 * (size_t)(triCount > 0 ? triCount : 0);
        }
        const size_t mbytes = dol_mask_words(w, h, d) * sizeof(uint32_t);
        const size_t ibytes = indices ? 3 * (size_t)triCount * sizeof(int) : 0;
        Dev dm(mbytes), dv(nv * sizeof(Vec3f)), di(ibytes);
        CheckCuda(cudaMemcpy(dm.p, mask, mbytes, cudaMemcpyHostToDevice), "copy to device");
        if (nv) CheckCuda(cudaMemcpy(dv.p, vertices, nv * sizeof(Vec3f), cudaMemcpyHostToDevice), "copy to device");
        if (ibytes) CheckCuda(cudaMemcpy(di.p, indices, ibytes, cudaMemcpyHostToDevice), "copy to device");
        const float bb[6] = {bbox.mMin.x, bbox.mMin.y, bbox.mMin.z, bbox.mMax.x, bbox.mMax.y, bbox.mMax.z};
        Check(dol_voxelize_triangles(triCount, static_cast<const int*>(di.p), static_cast<const float*>(dv.p), bb, w,
                                     h, d, static_cast<uint32_t*>(dm.p), nullptr));
        Check(dol_sync(nullptr));
        CheckCuda(cudaMemcpy(mask, dm.p, mbytes, cudaMemcpyDeviceToHost), "copy to host");
    }
}

#pragma GCC visibility pop
