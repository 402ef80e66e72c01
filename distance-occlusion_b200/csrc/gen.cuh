// gen.cuh -- synthetic input masks, in integer arithmetic so the host and the
// device produce the same bits.  These stand in for the inputs of the
// workloads the library is measured on; they are not part of the reference.
//
//   value noise : lattice spacing L, lattice values v in [0, 65536) from the
//                 reference's LCG (DistanceOcclusionLib.cpp:28-32) drawn x
//                 fastest, then y, then z; a voxel is set iff the trilinear
//                 interpolation at (x/L, y/L, z/L) is >= 1/2, evaluated exactly
//                 as sum(v * wx * wy * wz) >= 32768 * L^3.
//   shapes      : axis-aligned boxes and spheres with integer centres and
//                 sizes; a voxel is set iff its centre (x+1/2, y+1/2, z+1/2) is
//                 inside one of them (tests done on doubled coordinates).
#pragma once

#include "common.cuh"

namespace dolk {

DOL_HD uint32_t lcg_next(uint32_t s) { return s * 1103515245u + 12345u; }
DOL_HD int lcg_scale(uint32_t s, int limit) { return (int)(((uint64_t)s * (uint64_t)(uint32_t)limit) >> 32); }

struct NoiseSpec {
    int w, h, d, L, gx, gy, gz;   // lattice has gx*gy*gz points
    const uint16_t* lattice;      // [gz][gy][gx]
};

DOL_HD bool noise_bit(const NoiseSpec& s, int x, int y, int z)
{
    const int L = s.L;
    int i = x / L, j = y / L, k = z / L;
    uint32_t fx = (uint32_t)(x - i * L), fy = (uint32_t)(y - j * L), fz = (uint32_t)(z - k * L);
    uint64_t acc = 0;
    for (int c = 0; c < 8; c++) {
        int a = c & 1, b = (c >> 1) & 1, e = (c >> 2) & 1;
        uint32_t wx = a ? fx : (uint32_t)L - fx;
        uint32_t wy = b ? fy : (uint32_t)L - fy;
        uint32_t wz = e ? fz : (uint32_t)L - fz;
        uint32_t v = s.lattice[((size_t)(k + e) * s.gy + (j + b)) * s.gx + (i + a)];
        acc += (uint64_t)v * wx * wy * wz;
    }
    return acc >= (uint64_t)32768u * (uint64_t)(L * L * L);
}

// shape: kind 0 box (half sizes in doubled units), kind 1 sphere (radius)
struct Shape {
    int kind, cx, cy, cz, a, b, c;
};

DOL_HD bool shape_bit(const Shape* shapes, int n, int x, int y, int z)
{
    const long long px = 2 * x + 1, py = 2 * y + 1, pz = 2 * z + 1;
    for (int i = 0; i < n; i++) {
        const Shape& s = shapes[i];
        long long dx = px - 2LL * s.cx, dy = py - 2LL * s.cy, dz = pz - 2LL * s.cz;
        if (s.kind == 0) {
            // side a (x), b (y), c (z): centre +- side/2
            if (dx >= -s.a && dx < s.a && dy >= -s.b && dy < s.b && dz >= -s.c && dz < s.c) return true;
        } else {
            long long r2 = 4LL * s.a * s.a;
            if (dx * dx + dy * dy + dz * dz <= r2) return true;
        }
    }
    return false;
}

}  // namespace dolk
