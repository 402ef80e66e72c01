// k_sites.cu -- distances to float-positioned sites and their gradient.
//
// No reference counterpart: this extends the delta methods to differentiable
// sites without changing them.  Forward: each site marks the cell that holds
// it (an owner map keeps the smallest site index per cell), a delta method
// (Danielsson or JumpFlood, cw = 1) runs on that mask unchanged, and every
// cell p reads its owner through its delta and gets d_p = |p - site| in fp32,
// p being the cell centre.  Backward: with the owner assignment of the forward
// held fixed, dL/dsite_k = sum over cells owned by k of dL/dd_p *
// (site_k - p) / |site_k - p|.  Contributions are reduced per owner inside each
// warp (lanes with the same owner found with __match_any_sync, summed with
// shuffles), and one fp64 atomic per owner group scatters the partial sums;
// a last pass rounds them to fp32.  Per-cell directions are formed in fp64.
#include "common.cuh"
#include "kernels.h"

namespace dolk {

template <int kDim>
__global__ void k_sites_seed(int w, int h, int d, int n, const float* __restrict__ sites, uint32_t* __restrict__ mask,
                             int* __restrict__ cell_site)
{
    const int ws = words_per_row(w);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float sx = sites[kDim * i], sy = sites[kDim * i + 1], sz = kDim == 3 ? sites[kDim * i + 2] : 0.0f;
        int x = (int)floorf(sx), y = (int)floorf(sy), z = (int)floorf(sz);
        if (x < 0 || y < 0 || z < 0 || x >= w || y >= h || z >= d) continue;   // outside the grid: ignored
        long long row = (long long)z * h + y;
        atomicOr(mask + row * ws + (x >> 5), 1u << (x & 31));
        atomicMin(cell_site + row * w + x, i);
    }
}

template <int kDim>
__global__ void k_sites_forward(int w, int h, int d, int n, const void* __restrict__ deltas,
                                const int* __restrict__ cell_site, const float* __restrict__ sites,
                                int* __restrict__ owner, float* __restrict__ dist)
{
    const long long plane = (long long)w * h, cells = plane * d;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(c / plane);
        const long long r = c - z * plane;
        const int y = (int)(r / w), x = (int)(r - (long long)y * w);
        int tx, ty, tz = z;
        if (kDim == 2) {
            C2 dl = unpack2(static_cast<const uint32_t*>(deltas)[c]);
            tx = x + dl.x;
            ty = y + dl.y;
        } else {
            const int16_t* p = static_cast<const int16_t*>(deltas) + 3 * c;
            tx = x + p[0];
            ty = y + p[1];
            tz = z + p[2];
        }
        int k = -1;
        if (tx >= 0 && ty >= 0 && tz >= 0 && tx < w && ty < h && tz < d) {
            int v = cell_site[((long long)tz * h + ty) * w + tx];
            k = (v >= 0 && v < n) ? v : -1;   // cells without a site hold 0x7F7F7F7F
        }
        owner[c] = k;
        float dd = 0.0f;
        if (k >= 0) {
            float ex = sites[kDim * k] - ((float)x + 0.5f);
            float ey = sites[kDim * k + 1] - ((float)y + 0.5f);
            float s2 = __fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey));
            if (kDim == 3) {
                float ez = sites[kDim * k + 2] - ((float)z + 0.5f);
                s2 = __fadd_rn(s2, __fmul_rn(ez, ez));
            }
            dd = sqrtf(s2);
        } else {
            dd = __int_as_float(0x7fc00000);   // no site reachable: NaN
        }
        dist[c] = dd;
    }
}

template <int kDim>
__global__ void k_sites_backward(int w, int h, int d, const int* __restrict__ owner, const float* __restrict__ sites,
                                 const float* __restrict__ grad_dist, double* __restrict__ acc)
{
    const long long plane = (long long)w * h, cells = plane * d;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long start = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    // every lane of a warp runs the same number of iterations so the warp
    // collectives below always see all 32 lanes
    const long long span = (cells + stride - 1) / stride;
    for (long long it = 0; it < span; it++) {
        const long long c = start + it * stride;
        int k = -1;
        double g[3] = {0.0, 0.0, 0.0};
        if (c < cells) {
            k = owner[c];
            if (k >= 0) {
                const int z = (int)(c / plane);
                const long long r = c - z * plane;
                const int y = (int)(r / w), x = (int)(r - (long long)y * w);
                // direction in fp64: the per-cell unit vectors of a site largely
                // cancel in the sum, so their rounding is kept well below 1e-5
                double e[3];
                e[0] = (double)sites[kDim * k] - ((double)x + 0.5);
                e[1] = (double)sites[kDim * k + 1] - ((double)y + 0.5);
                e[2] = kDim == 3 ? (double)sites[kDim * k + 2] - ((double)z + 0.5) : 0.0;
                const double len = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
                const float gd = grad_dist[c];
                if (len > 0.0 && gd == gd) {
                    const double sc = (double)gd / len;
                    for (int a = 0; a < kDim; a++) g[a] = sc * e[a];
                } else {
                    k = -1;   // the gradient of |p - s| is undefined at the site itself
                }
            }
        }
        // segmented reduce within the warp: lanes that share an owner
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, k);
        const int leader = __ffs(peers) - 1;
        double sum[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < kDim; a++) {
            double v = g[a];
            // sum over the peer group: every lane adds the values of its peers
            double tot = 0.0;
            unsigned m = peers;
            while (m) {
                const int src = __ffs(m) - 1;
                m &= m - 1;
                tot += __shfl_sync(peers, v, src);
            }
            sum[a] = tot;
        }
        if (k >= 0 && lane == leader)
            for (int a = 0; a < kDim; a++) atomicAdd(acc + (long long)kDim * k + a, sum[a]);
    }
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)a[i];
}

static int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    long long cap = (long long)g_num_sms * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

void launch_sites_seed(int dim, int w, int h, int d, int n, const float* sites, uint32_t* mask, int* cell_site,
                       cudaStream_t st)
{
    ProfScope ps("sites_seed", st);
    const long long cells = (long long)w * h * d;
    cudaMemsetAsync(mask, 0, (size_t)words_per_row(w) * h * d * sizeof(uint32_t), st);
    cudaMemsetAsync(cell_site, 0x7F, (size_t)cells * sizeof(int), st);   // 0x7F7F7F7F > any site index
    if (dim == 2)
        k_sites_seed<2><<<grid_for(n, 256), 256, 0, st>>>(w, h, d, n, sites, mask, cell_site);
    else
        k_sites_seed<3><<<grid_for(n, 256), 256, 0, st>>>(w, h, d, n, sites, mask, cell_site);
}

void launch_sites_forward(int dim, int w, int h, int d, int n, const void* deltas, const int* cell_site,
                          const float* sites, int* owner, float* dist, cudaStream_t st)
{
    ProfScope ps("sites_forward", st);
    const long long cells = (long long)w * h * d;
    if (dim == 2)
        k_sites_forward<2><<<grid_for(cells, 256), 256, 0, st>>>(w, h, d, n, deltas, cell_site, sites, owner, dist);
    else
        k_sites_forward<3><<<grid_for(cells, 256), 256, 0, st>>>(w, h, d, n, deltas, cell_site, sites, owner, dist);
}

void launch_sites_backward(int dim, int w, int h, int d, int n, const int* owner, const float* sites,
                           const float* grad_dist, double* acc, float* grad_sites, cudaStream_t st)
{
    ProfScope ps("sites_backward", st);
    const long long cells = (long long)w * h * d;
    cudaMemsetAsync(acc, 0, (size_t)n * dim * sizeof(double), st);
    if (dim == 2)
        k_sites_backward<2><<<grid_for(cells, 256), 256, 0, st>>>(w, h, d, owner, sites, grad_dist, acc);
    else
        k_sites_backward<3><<<grid_for(cells, 256), 256, 0, st>>>(w, h, d, owner, sites, grad_dist, acc);
    k_to_float<<<grid_for((long long)n * dim, 256), 256, 0, st>>>(acc, grad_sites, (long long)n * dim);
}

}  // namespace dolk
