// Heightmap voxeliser on the GPU: GeometryEngine::getGroundHeight
// (06_transient_localization_dx1.cpp:144-192) for every column of the grid,
// one thread per column.  Compiled with -fmad=false, so each FP64 expression
// is rounded exactly as the host's (built with -ffp-contract=off, same
// operation order): the ground heights, and with them the mask, are
// bit-identical to HeightField::ground_height.  The ray cast is
// O(columns x triangles per bin); a city mesh of millions of triangles makes
// it the dominant set-up cost on the host.
#include <cuda_runtime.h>

#include <vector>

#include "geometry.hpp"

namespace lbm {
namespace {

constexpr int kBinRows = 200, kBinCols = 200;   // GeometryEngine::gridRows/gridCols (06:66)

struct GridView
{
    const double* tri;   // [n][15]: v1, v2, v3, min, max
    const int* start;    // CSR offsets, kBinRows * kBinCols + 1
    const int* items;
    double gmin0, gmin1, gmax0, gmax1, cell_w, cell_h;
    int ntris;
};

__device__ double column_height(const GridView& g, double x, double y)
{
    if (g.ntris == 0) return -1e30;
    if (x < g.gmin0 || x > g.gmax0 || y < g.gmin1 || y > g.gmax1) return -1e30;
    const int r = (int)((x - g.gmin0) / g.cell_w);
    const int c = (int)((y - g.gmin1) / g.cell_h);
    if (r < 0 || r >= kBinRows || c < 0 || c >= kBinCols) return -1e30;
    const int b = r * kBinCols + c;
    // Moller-Trumbore, ray origin (x, y, 10000), direction (0, 0, -1), EPS 1e-9.
    const double ro[3] = {x, y, 10000.0};
    const double rd[3] = {0.0, 0.0, -1.0};
    const double EPS = 1e-9;
    double max_z = -1e30;
    for (int n = g.start[b]; n < g.start[b + 1]; ++n)
    {
        const double* t = g.tri + 15 * (size_t)g.items[n];
        const double *v1 = t, *v2 = t + 3, *v3 = t + 6, *mn = t + 9, *mx = t + 12;
        if (mx[0] < x - 1e-6 || mn[0] > x + 1e-6) continue;
        if (mx[1] < y - 1e-6 || mn[1] > y + 1e-6) continue;
        const double e1[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
        const double e2[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
        const double h[3] = {rd[1] * e2[2] - rd[2] * e2[1], rd[2] * e2[0] - rd[0] * e2[2], rd[0] * e2[1] - rd[1] * e2[0]};
        const double a = e1[0] * h[0] + e1[1] * h[1] + e1[2] * h[2];
        if (fabs(a) < EPS) continue;
        const double f = 1.0 / a;
        const double s[3] = {ro[0] - v1[0], ro[1] - v1[1], ro[2] - v1[2]};
        const double u = f * (s[0] * h[0] + s[1] * h[1] + s[2] * h[2]);
        if (u < 0.0 || u > 1.0) continue;
        const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
        const double v = f * (rd[0] * q[0] + rd[1] * q[1] + rd[2] * q[2]);
        if (v < 0.0 || (u + v) > 1.0) continue;
        const double tt = f * (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]);
        if (tt > EPS)
        {
            const double hit = ro[2] + tt * rd[2];
            if (hit > max_z) max_z = hit;
        }
    }
    return max_z;
}

__global__ void __launch_bounds__(128) k_ground_height(GridView g, double x_min, double y_min, double dx, int nxt,
                                                       int nyt, double* __restrict__ gH)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nxt) return;
    // cell centre of halo-inclusive column (i, j) (06:464-465)
    const double x = x_min + ((i - 1) + 0.5) * dx;
    const double y = y_min + ((j - 1) + 0.5) * dx;
    gH[(size_t)j * nxt + i] = column_height(g, x, y);
}

}  // namespace

int ground_height_device(const HeightField& geo, double x_min, double y_min, double dx, int nxt, int nyt,
                         double* gH, void* stream_p)
{
    cudaStream_t stream = (cudaStream_t)stream_p;
    std::vector<double> tri;
    std::vector<int> start, items;
    double gmin[3], gmax[3], cw, ch;
    geo.export_flat(tri, start, items, gmin, gmax, cw, ch);
    if (start.empty()) start.assign((size_t)kBinRows * kBinCols + 1, 0);
    double *d_tri = nullptr, *d_gH = nullptr;
    int *d_start = nullptr, *d_items = nullptr;
    const size_t ncol = (size_t)nxt * nyt;
    cudaError_t e = cudaMalloc(&d_tri, std::max<size_t>(tri.size(), 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_start, start.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_items, std::max<size_t>(items.size(), 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_gH, ncol * sizeof(double));
    if (e == cudaSuccess && !tri.empty())
        e = cudaMemcpyAsync(d_tri, tri.data(), tri.size() * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
    {
        GridView g{d_tri, d_start, d_items, gmin[0], gmin[1], gmax[0], gmax[1], cw, ch, (int)geo.triangle_count()};
        k_ground_height<<<dim3((unsigned)((nxt + 127) / 128), (unsigned)nyt), 128, 0, stream>>>(g, x_min, y_min, dx,
                                                                                                 nxt, nyt, d_gH);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(gH, d_gH, ncol * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_tri);
    cudaFree(d_start);
    cudaFree(d_items);
    cudaFree(d_gH);
    return (int)e;
}

}  // namespace lbm
