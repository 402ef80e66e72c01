/*
 * ref_mesh.cpp -- C entry points into the UNMODIFIED reference voxeliser.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file
 * into oracle/_ref/libdolref.so with -I pointing at the reference checkout;
 * it includes MeshSupport.cpp exactly as it lies there.  A translation unit
 * of its own: MeshSupport.cpp opens namespace MSL at file scope.
 */
#include <stdint.h>   /* MeshSupport.h uses uint32_t; the tool includes it after stdint */
#include "MeshSupport.cpp"

extern "C" {

/* MSL::CreateBitMaskFromTriangles (MeshSupport.cpp:369-475): ORs the cells
 * the triangles touch into mask.  bbox: min x, y, z, max x, y, z.  The
 * reference dereferences indices unconditionally, so they are required. */
void ref_voxelize(int tri_count, const int* indices, const float* vertices, const float* bbox, int w, int h, int d,
                  uint32_t* mask)
{
    Bounds3f b = {{bbox[0], bbox[1], bbox[2]}, {bbox[3], bbox[4], bbox[5]}};
    CreateBitMaskFromTriangles(tri_count, indices, reinterpret_cast<const Vec3f*>(vertices), b, w, h, d, mask);
}

}  /* extern "C" */
