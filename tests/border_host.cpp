// Host build of the border-initialisation gather (csrc/border.cuh) for the CPU
// tests: the same __host__ __device__ code the CUDA kernel runs, compiled with
// g++ and exposed through a C entry point that fills a whole delta array.
#include "border.cuh"

extern "C" void host_border_2d(int w, int h, const uint32_t* mask, int16_t* out)
{
    const int ws = dolk::words_per_row(w);
    for (int y = 0; y < h; y++)
        for (int k = 0; k < ws; k++) {
            dolk::Planes2 p = dolk::border2_word(w, h, mask, y, k);
            for (int b = 0; b < 32 && 32 * k + b < w; b++) {
                dolk::C2 c = dolk::decode2(p, b);
                size_t i = 2 * ((size_t)y * w + 32 * k + b);
                out[i] = (int16_t)c.x;
                out[i + 1] = (int16_t)c.y;
            }
        }
}

extern "C" void host_border_3d(int w, int h, int d, const uint32_t* mask, int16_t* out)
{
    const int ws = dolk::words_per_row(w);
    for (int z = 0; z < d; z++)
        for (int y = 0; y < h; y++)
            for (int k = 0; k < ws; k++) {
                dolk::Planes3 p = dolk::border3_word(w, h, d, mask, z, y, k);
                for (int b = 0; b < 32 && 32 * k + b < w; b++) {
                    dolk::C3 c = dolk::decode3(p, b);
                    size_t i = 3 * (((size_t)z * h + y) * w + 32 * k + b);
                    out[i] = (int16_t)c.x;
                    out[i + 1] = (int16_t)c.y;
                    out[i + 2] = (int16_t)c.z;
                }
            }
}
