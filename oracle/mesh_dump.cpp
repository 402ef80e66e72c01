/*
 * mesh_dump.cpp -- reads an OBJ file with the reference's own reader and
 * bounds (MSL::ReadObjFile, MSL::FindBounds; MeshSupport.cpp:795-868) and
 * writes the triangles the reference tool would voxelise
 * (DistanceOcclusionTool.cpp:905-934) as a flat binary file:
 *     int32 tri_count, int32 vertex_count, float bbox[6] (min xyz, max xyz),
 *     float vertices[3 * vertex_count], int32 indices[3 * tri_count]
 * TEST INFRASTRUCTURE ONLY: oracle/Makefile runs it on the reference's sample
 * mesh so that the GPU tests can use it where the reference checkout is absent.
 */
#include <stdint.h>   /* MeshSupport.h uses uint32_t; the tool includes it after stdint */
#include "MeshSupport.cpp"

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: mesh_dump in.obj out.tri\n");
        return 1;
    }
    FILE* in = fopen(argv[1], "r");
    if (!in) return 1;
    cMesh mesh;
    const bool ok = ReadObjFile(in, &mesh);
    fclose(in);
    if (!ok) return 1;
    const Bounds3f b = FindBounds(mesh);
    const int tris = (int)mesh.mPositionIndices.size() / 3, verts = (int)mesh.mPositions.size();
    FILE* out = fopen(argv[2], "wb");
    if (!out) return 1;
    const float bb[6] = {b.mMin.x, b.mMin.y, b.mMin.z, b.mMax.x, b.mMax.y, b.mMax.z};
    fwrite(&tris, 4, 1, out);
    fwrite(&verts, 4, 1, out);
    fwrite(bb, 4, 6, out);
    fwrite(mesh.mPositions.data(), 12, verts, out);
    fwrite(mesh.mPositionIndices.data(), 4, 3 * (size_t)tris, out);
    fclose(out);
    return 0;
}
