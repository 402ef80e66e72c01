// MeshSupportB200.h -- the voxeliser of the reference's MeshSupport.h
// (namespace MSL, CreateBitMaskFromTriangles) on the GPU, for host code that
// voxelises meshes.  Same types and signature: a caller that links this
// library instead of compiling MeshSupport.cpp's voxeliser gets the same
// bits.  Arrays are HOST memory; each call copies them to the device, runs
// dol_voxelize_triangles (dol_b200.h) and copies the mask back.  Failures
// throw DOL::Error.
#ifndef MESH_SUPPORT_B200_H
#define MESH_SUPPORT_B200_H

#include <stdint.h>

namespace MSL
{
    struct Vec3f { float x; float y; float z; };
    struct Bounds3f { Vec3f mMin; Vec3f mMax; };

    void CreateBitMaskFromTriangles
    (
        int             triCount,
        const int       indices[],     // NULL: vertices three per triangle
        const Vec3f     vertices[],
        const Bounds3f& bbox,
        int w, int h, int d,
        uint32_t        mask[]         // ORed into, as the reference does
    );
}

#endif
