// Device-side data layout and kernel launchers of the D3Q19 acoustic step.
// Included by the host C++ (api.cpp, built with g++) and by kernels.cu.
//
// Population layout in HBM: block-interleaved ("array of structures of
// arrays").  Each row (j, k) of the halo-inclusive grid, j = 0..ny+1,
// k = 0..nz+1 (06:206-209), holds nb = ceil(nx/bc) blocks of bc cells along
// x, bc = 128 bytes / element size (32 FP32 or 64 FP16 cells); a block
// stores its 19 directions one after the other, bc elements each, so every
// direction of a block is exactly one 128-byte line:
//     elem(q, i, j, k) = kFrontElems + (k * (ny+2) + j) * row_stride
//                        + ((i-1) / bc) * 19 bc + q * bc + ((i-1) % bc)
// for interior columns i = 1..nx, with row_stride = nb * 19 bc.  A thread's
// 19 loads or stores for one row therefore differ by compile-time
// immediates (q * bc), and a warp-wide access of one direction reads or
// writes whole lines.  The x-halo columns are not stored: open x
// faces keep their ghosts in the compact x-face buffers (XFace).
// Stored values are deviations from rest equilibrium, g_q = f_q - w_q, times
// `scale` (1 for FP32; the per-run FP16 scale otherwise).
//
// Per-cell side arrays (links words, near-solid bits) use a plain padded
// layout: cell(i, j, k) = k * plane + j * pitch + (i - 1).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "check.cuh"
#include "nlos_lbm.h"

namespace lbm {

constexpr int kMaxSources = 8;
constexpr int kLineBytes = 128;
// cells per interleaved block for an element size in bytes (one line per direction)
__host__ __device__ constexpr int block_cells(int esz) { return kLineBytes / esz; }
constexpr long long kFrontElems = 19 * 64 + 64;   // pad before the first row (>= one block)
constexpr long long kBackElems = 19 * 64 + 64;    // pad after the last row

struct Layout
{
    int nx, ny, nz;          // interior cells
    int pitch;               // x pitch of the side arrays, round_up(nx + 2, 32)
    int words_per_row;       // pitch / 32 (near-solid bitmap)
    long long plane;         // pitch * (ny + 2)
    int bc;                  // cells per interleaved block (32 FP32, 64 FP16)
    int bc_shift;            // log2(bc)
    int nb;                  // blocks per row
    long long row_stride;    // nb * 19 * bc population elements per row
    long long plane_stride;  // (ny + 2) * row_stride
    long long total;         // population elements per buffer, pads included

    __host__ __device__ long long cell(int i, int j, int k) const
    {
        return (long long)k * plane + (long long)j * pitch + (i - 1);
    }
    __host__ __device__ long long elem(int q, int i, int j, int k) const
    {
        const int c = i - 1;
        return kFrontElems + ((long long)k * (ny + 2) + j) * row_stride +
               (long long)(c >> bc_shift) * (19 * bc) + q * bc + (c & (bc - 1));
    }
};

// Device control block: read by the kernels of a batched (graph) step.
struct Control
{
    long long step;        // time step index of the step being executed
    long long table_base;  // step index of source-table row 0
    long long probe_base;  // step index of probe-buffer row 0
    int nonfinite;         // set by the probe kernels when an owned probe reads a non-finite value
                           // (the host uploads only the fields above it)
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
    double wsum;           // > 0: fluid weight sum of the whole stencil, given by the host when the
                           // stencil reaches past this z-slab (0: the kernel sums its own cells)
};

struct SourceArgs
{
    int nsrc;
    SourceStatic st[kMaxSources];
    SourceEntry direct[kMaxSources];   // used when table == nullptr
    const SourceEntry* table;          // [row][nsrc], row = step - ctl->table_base
    const Control* ctl;                // nullptr: use `direct`
    double x_min, y_min, z_min, dx;   // origin of the whole grid
    float scale;
    int k_off;                         // first z-layer of this handle's slab (0: the whole grid)
};

struct GhostFace
{
    int axis, side;        // 0/1/2, 0 low / 1 high
    int nu, nv;            // tangential interior extents
    long long first;       // first thread index of this face
};

// x-face buffers (float, stored deviation units).  The fused step exports
// the post-collision populations of the cells next to the x faces into
// `xexp`, the ghost kernel turns them into the open-boundary ghosts `xgh`,
// and the step reads those for the first and last cell of each row.  Both
// are [side][q][k][j], coalesced along j.
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
    float4* face_mom;          // non-null: moments (rho', J) of each ghost's interior cell, [total]
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
};

struct ProbeArgs
{
    int n;
    const int* ijk;            // [n][3] halo-inclusive cell coordinates; i = -1: not owned
    double* out;               // [row][n], row = step - probe_base
    double* energy;            // [n] running sum of p^2 (FP64)
    Control* ctl;              // nullptr: row = direct_row, no counter update
    long long direct_row;
    float scale;
    int* nonfinite;            // set to 1 when an owned probe reads a non-finite value
};

// Scheme A (the reference's 01-04 family).  The stored state is the
// post-collision populations P^s as deviations from the background
// equilibrium feq(1, u0) (so a uniform flow is an exact fixed point and FP32
// resolves the acoustic perturbation, not the flow); a step pulls P^s (pull = stream of the
// source cells' post-collision values), adds the destination source,
// collides with the cell's own omega and stores P^{s+1}.  A population that
// arrives from a SOLID cell must be the destination's own pre-collision value
// of the opposite direction: each fluid cell writes that value into the
// SOLID neighbour's (otherwise unused) slot for the next step, so the next
// pull reads it like any other.  Zero-gradient halos are collided copies of
// the nearest interior cell, written for the next step by k_copy_a.  x-halo
// values live in two x-face arrays that alternate with the step parity.
struct SchemeAArgs
{
    const float* om_x;         // 1/tau per interior column i-1 (tau ramp), likewise om_y, om_z;
    const float* om_y;         //   a cell's omega is the minimum of the three
    const float* om_z;
    float om_bulk;             // 1/tau of halo cells (they lie outside every ramp)
    const float* fld_x;        // source weight factors, halo-inclusive index 0..n+1;
    const float* fld_y;        //   weight(i,j,k) = fld_x[i] fld_y[j] fld_z[k]
    const float* fld_z;
    int field_mode;            // -1: no field source, 0: LBM_FIELD_DST, 1: LBM_FIELD_FORCE, 2: LBM_FIELD_PRE
    int src_index;             // which source of the schedule is the field source
    int nsrc;
    float flow[3];             // background velocity u0 (lattice units)
    float base[19];            // feq(1, u0) - w_q: stored values are deviations from feq(1, u0)
    float cu0[19];             // c_q . u0
    float fq[19];              // w_q (1 + 3 c_q . u0): forcing weight of direction q (03:74-78)
    float u0sq;                // u0 . u0
    const SourceEntry* table;  // schedule rows [row][nsrc] (row = step - ctl->table_base), as SourceArgs
    const Control* ctl;        // nullptr: use mass_direct
    float mass_direct[2];      // mass of step s and of step s + 1 (direct launches)
    float* xgh_out;            // x-halo values written for the next step
    int copy;                  // zero-gradient halos on every face
    const float* sg_x;         // destination blend toward rest (01:207-225, 01:343-347): strength per
    const float* sg_y;         //   interior column i-1, likewise sg_y, sg_z; a cell's is the maximum
    const float* sg_z;         //   of the three, 0 outside the layer
    int blend;                 // 1: populations that left a fluid cell are blended, (1-s) f + s w_q
    int zper;                  // 1: periodic z, halo planes 0 / nz+1 repeat planes nz / 1
    const float* sg_xy;        // nullptr or per-column blend strengths [(j-1) nx + (i-1)] (max with sg_*)
    const float* fld_xy;       // nullptr or per-column source weights, replacing fld_x fld_y fld_z
    int nx_col, ny_col;        // column grid of sg_xy / fld_xy (nx, ny)
    int prefetch_rows;         // > 0: the instance with per-column fields (04's) prefetches into L2 the
                               //   storage row first read this many rows ahead
};

// ---- launchers (kernels.cu) ----------------------------------------------
// storage: 0 = float, 1 = __half.  All launches go to `stream`.
cudaError_t launch_build_links(const uint8_t* mask_ref, uint32_t* links, uint32_t* near, const Layout& L,
                               cudaStream_t stream);
cudaError_t launch_source(int storage, void* f, const Layout& L, const StepArgs& sa, const SourceArgs& a,
                          cudaStream_t stream);
cudaError_t launch_ghost(int storage, void* f, const Layout& L, const GhostArgs& a, cudaStream_t stream);
// Fused step: FP32 storage runs the two-cells-per-thread pair kernel, FP16
// storage the warp pipelines of cp.async copies.
cudaError_t launch_step(int storage, const void* fin, void* fout, const Layout& L, const StepArgs& a,
                        float scale, cudaStream_t stream);
// One-time set-up of the fused step on the current device (shared-memory
// attribute, occupancy); call before the first launch or capture.
cudaError_t prepare_step(int storage);
// Fused step (FP32 storage, the default implementation) that also writes the
// moments (rho', jx, jy, jz) of every cell's pulled populations to `mom`: the
// forward data of the adjoint's BGK Jacobian, where they enter only through
// terms of the wave's amplitude (J^2, J / r, 1 / r with r = 1 + rho').  Each
// value is kept as a 12-bit float (sign, FP16's 5-bit exponent, 6 mantissa
// bits: FP16 rounded to nearest-even at its 4 lowest mantissa bits), the two
// cells of an x pair (c, c + 1), c even, in one PairMoments of 96 bits, values
// v0..v7 = rho', jx, jy, jz of cell c then of cell c + 1, v_i at bits 12 i;
// pairs in dense order ((k-1) ny + (j-1)) ceil(nx / 2) + c / 2.  That is 6
// bytes per cell, so most of a long run's moments stay in memory instead of
// being recomputed, at a rounding step (2^-7) that moves the gradient far
// less than the 1e-4 bar (8-bit floats, 2^-3, came within 12 % of it).
struct PairMoments
{
    unsigned w[3];
};
cudaError_t launch_step_moments(const float* fin, float* fout, const Layout& L, const StepArgs& a,
                                PairMoments* mom, cudaStream_t stream);
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

// Scheme A: fused step (FP32 storage), the zero-gradient halo copies of the
// next step, the initial state, and probes / field of a scheme-A state.
cudaError_t launch_step_a(const float* fin, float* fout, const Layout& L, const StepArgs& a, const SchemeAArgs& b,
                          cudaStream_t stream);
cudaError_t launch_copy_a(const float* fin, float* fout, const Layout& L, const StepArgs& a, const SchemeAArgs& b,
                          cudaStream_t stream);
cudaError_t launch_init_a(float* f0, float* f1, float* xgh0, float* xgh1, const uint8_t* mask_ref, const Layout& L,
                          const SchemeAArgs& b, cudaStream_t stream);
cudaError_t launch_probe_a(const float* f, const Layout& L, const StepArgs& sa, const SchemeAArgs& b,
                           const ProbeArgs& a, cudaStream_t stream);
cudaError_t launch_field_rho_a(const float* f, float* out, const Layout& L, const StepArgs& sa, const SchemeAArgs& b,
                               cudaStream_t stream);
// Periodic z: copy the stored values of the FLUID cells of planes nz and 1
// into halo planes 0 and nz + 1 (a SOLID cell's slots are its mailbox), for
// the initial state; the step kernel stores those planes twice itself.
cudaError_t launch_zper_a(float* f, const Layout& L, const StepArgs& sa, cudaStream_t stream);
// Initial state at rest with density 1 + rho_prime (interior cells, x
// fastest) over the state lbm_init left: FLUID interior cells and the slots
// of SOLID cells next to them.  mask_ref: the halo-inclusive mask.
cudaError_t launch_set_density_a(float* f, float* xgh, const float* rho_prime, const uint8_t* mask_ref,
                                 const Layout& L, const SchemeAArgs& b, cudaStream_t stream);

// z-slab messages: the 5 crossing directions of one plane as whole lines plus
// its two crossing x-face ghost rows (kernels.cu); pack: plane k -> msg,
// otherwise msg -> plane k.  up: the directions with ez = +1 (else -1).
long long slab_message_bytes(const Layout& L);
cudaError_t launch_slab_msg(bool pack, void* f, float* xgh, void* msg, const Layout& L, int k, int up, int esz,
                            cudaStream_t stream);

// Bounds-checked builds (-DLBM_CHECK): read and clear the first failed check
// of each kernel file (site 0: none; always 0 in the product build), and a
// kernel that fails one check on purpose (site 99) without touching memory.
cudaError_t check_read_kernels(check::Status* out);
cudaError_t check_read_adjoint(check::Status* out);
cudaError_t check_read_scheme_a(check::Status* out);
cudaError_t launch_check_selftest(cudaStream_t stream);

// Capacity (cells) of the statically reserved field array used by
// lbm_get_rho_noalloc, and the device address of that array on `device`
// (looked up on first use with the device current; must not run during
// stream capture).
constexpr long long kNoAllocFieldCells = LBM_NOALLOC_MAX_CELLS;   // 2^23 floats = 32 MiB, the API's limit
constexpr int kMaxDevices = 64;
cudaError_t field_scratch_address(int device, float** ptr);

}  // namespace lbm
