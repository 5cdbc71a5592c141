// Device-side data layout and kernel launchers of the D3Q19 acoustic step.
// Included by the host C++ (api.cpp, built with g++) and by kernels.cu.
//
// Population layout in HBM (structure of arrays, one array per direction q):
//   element (i, j, k) of direction q, in the reference's halo-inclusive cell
//   coordinates i = 0..nx+1, j = 0..ny+1, k = 0..nz+1 (06:206-209), lives at
//       base + q * pop_stride + k * plane + j * pitch + (i - 1)
//   pitch = round_up(nx + 2, 32), plane = pitch * (ny + 2).
//   Interior rows therefore start on a 128-byte (FP32) / 64-byte (FP16)
//   boundary, the x-high halo sits at column nx, and the x-low halo of row j
//   occupies the last (padding) column of row j-1; one 32-element pad before
//   the origin holds the x-low halo of (j=0, k=0).  Pull offsets are the same
//   for every cell: src = dst - (ex + ey * pitch + ez * plane).
// Stored values are deviations from rest equilibrium, g_q = f_q - w_q, times
// `scale` (1 for FP32; the per-run FP16 scale otherwise).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace lbm {

constexpr int kMaxSources = 8;
constexpr int kFrontPad = 32;
// Elements after the last plane: a staged row copy of the last row may run
// up to one tile (<= 512 elements) plus its alignment margin past it.
constexpr int kBackPad = 1024;

struct Layout
{
    int nx, ny, nz;        // interior cells
    int pitch;             // x pitch, elements
    int words_per_row;     // pitch / 32 (near-solid bitmap)
    long long plane;       // pitch * (ny + 2)
    long long pop_stride;  // elements per direction array, incl. pads
    // Linear cell index of halo-inclusive coordinates (relative to the origin).
    long long cell(int i, int j, int k) const { return (long long)k * plane + (long long)j * pitch + (i - 1); }
};

// Device control block: read by the kernels of a batched (graph) step.
struct Control
{
    long long step;        // time step index of the step being executed
    long long table_base;  // step index of source-table row 0
    long long probe_base;  // step index of probe-buffer row 0
};

struct SourceStatic
{
    int injection;         // LBM_INJECT_*
    int radius;            // Gaussian stencil radius
    double sigma2;         // (sigma_cells * dx)^2
};

struct SourceEntry
{
    double cx, cy, cz;     // position at this step (DroneSource::update, 06:221-238)
    double mass;           // val(t) * dt * gain: total mass injected this step (06:631)
};

struct SourceArgs
{
    int nsrc;
    SourceStatic st[kMaxSources];
    SourceEntry direct[kMaxSources];   // used when table == nullptr
    const SourceEntry* table;          // [row][nsrc], row = step - ctl->table_base
    const Control* ctl;                // nullptr: use `direct`
    double x_min, y_min, z_min, dx;
    float scale;
};

struct GhostFace
{
    int axis, side;        // 0/1/2, 0 low / 1 high
    int nu, nv;            // tangential interior extents
    long long first;       // first thread index of this face
};

// x-face buffers (float, stored deviation units).  The x-halo columns of the
// population arrays are not used: the fused step exports the post-collision
// populations of the cells next to the x faces into `xexp`, the ghost kernel
// turns them into the open-boundary ghosts `xgh`, and the step reads those
// for the first and last cell of each row.  Both are [side][q][k][j] and
// coalesced along j, so no strided column of the populations is touched.
//   xexp: side 0/1 = cells i = 1 / i = nx, j = 1..ny, k = 1..nz  -> [2][Q][nz][ny]
//   xgh : side 0/1 = halo i = 0 / i = nx+1, j = 0..ny+1, k = 0..nz+1 -> [2][Q][nz+2][ny+2]
struct XFace
{
    float* xexp;
    float* xgh;
    __host__ __device__ long long exp_index(int side, int q, int j, int k, int ny, int nz) const
    {
        return ((long long)(side * 19 + q) * nz + (k - 1)) * ny + (j - 1);
    }
    __host__ __device__ long long gh_index(int side, int q, int j, int k, int ny, int nz) const
    {
        return ((long long)(side * 19 + q) * (nz + 2) + k) * (ny + 2) + j;
    }
};

struct GhostArgs
{
    int nfaces;
    GhostFace face[6];
    long long total;
    float scale;
    XFace xf;
};

struct StepArgs
{
    const uint32_t* links;     // per cell; only read where the near bit is set
    const uint32_t* near;      // 1 bit per interior cell: SOLID or a SOLID neighbour
    const float* sig_x;        // per-axis sponge strength, index = interior i-1, j-1, k-1
    const float* sig_y;
    const float* sig_z;
    float omega;               // 1 / tau
    XFace xf;
    // Per direction, in elements (warp-uniform address offsets):
    long long pull_off[19];    // q * pop_stride - (ey * pitch + ez * plane): aligned source of a pair
    long long pop_off[19];     // q * pop_stride
    int* error;                // set when a bounded wait in a kernel gives up (0 = fine)
    int prefetch_rows;         // > 0: each block prefetches into L2 the source rows of the row this far ahead
};

// Error codes a kernel writes to StepArgs::error.
constexpr int kErrStageTimeout = 1;   // staged-copy barrier wait exceeded its limit

struct ProbeArgs
{
    int n;
    const long long* cell;     // linear index, -1 = not owned
    double* out;               // [row][n], row = step - probe_base
    double* energy;            // [n] running sum of p^2 (FP64)
    Control* ctl;              // nullptr: row = direct_row, no counter update
    long long direct_row;
    float scale;
};

// ---- launchers (kernels.cu) ----------------------------------------------
// storage: 0 = float, 1 = __half.  All launches go to `stream`.
cudaError_t launch_build_links(const uint8_t* mask_ref, uint32_t* links, uint32_t* near, const Layout& L,
                               cudaStream_t stream);
cudaError_t launch_source(int storage, void* f, const Layout& L, const StepArgs& sa, const SourceArgs& a,
                          cudaStream_t stream);
cudaError_t launch_ghost(int storage, void* f, const Layout& L, const GhostArgs& a, cudaStream_t stream);
// variant: implementation / launch shape of the fused step; all do the same
// work.  0-3: register-resident pairs with lane shuffles (0: 128 threads,
// 1: 128 threads with at most 64 registers, 2: 256 threads, 3: 64 threads);
// 4-7: persistent CTAs staging rows in shared memory with bulk async copies
// (tile width / stages 256/3, 256/2, 128/4, 512/2); 8, 9: four cells per
// thread with 8-byte vectors (FP16 storage; 9 caps registers at 80; FP32
// storage runs variant 3); 10-12: pair kernel with 32-bit per-thread offsets
// (128 threads, 128 threads with at most 64 registers, 64 threads).  `grid` is the persistent
// grid from prepare_step (ignored by 0-3).
cudaError_t launch_step(int storage, const void* fin, void* fout, const Layout& L, const StepArgs& a,
                        float scale, int variant, int grid, cudaStream_t stream);
// Per-variant set-up (shared-memory opt-in, persistent grid size); call
// once per device before the first launch and outside stream capture.
cudaError_t prepare_step(int storage, int variant, int device, int* grid);
cudaError_t launch_probe(int storage, const void* f, const Layout& L, const StepArgs& sa, const ProbeArgs& a,
                         cudaStream_t stream);
// (float)(rho - 1) of every interior cell, pulled from the pre-step buffer `f`.
cudaError_t launch_field_rho(int storage, const void* f, float* out, const Layout& L, const StepArgs& sa,
                             float scale, cudaStream_t stream);
// Conversions between the stored deviations and FP64 f in the reference's
// AoS halo-inclusive layout (f[idx*19+q]).
cudaError_t launch_export_f(int storage, const void* f, double* out, const Layout& L, const XFace& xf, float scale,
                            cudaStream_t stream);
cudaError_t launch_import_f(int storage, void* f, const double* in, const Layout& L, const XFace& xf, float scale,
                            cudaStream_t stream);

}  // namespace lbm
