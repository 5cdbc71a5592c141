// C-ABI of the B200 D3Q19 acoustic solver (include/nlos_lbm.h).
//
// Host side of LBMSolver (06_transient_localization_dx1.cpp:241-1122): the
// grid/mask/sponge/probe set-up of init() and the source schedule of
// apply_source() are computed here in FP64 exactly as the reference does; the
// per-cell work runs in the sm_100a kernels of kernels.cu.  Compiled with
// -ffp-contract=off so the FP64 host arithmetic keeps the reference's
// rounding.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "adjoint.hpp"
#include "device.hpp"
#include "geometry.hpp"
#include "lattice.cuh"
#include "nlos_lbm.h"

using namespace lbm;

namespace {

constexpr int kTableRows = 4096;   // source-schedule rows resident on the device
constexpr int kBcCut = 100;        // face of a z-slab that borders the next slab (internal face type)
constexpr int kProbeRows = 4096;   // probe-series rows buffered on the device
// L2 prefetch distance of the adjoint step in rows (measured on the 256x256x128 patch: 192 rows
// ahead; per-line prefetches gave 2-4 % less time per gradient than none, 48 to 1536 rows tried,
// and one bulk prefetch of the whole storage row 4 % more)
constexpr int kDefaultAdjointPrefetchRows = 192;
// The same for the scheme-A instance with per-column fields, latency-bound like the adjoint step
// (04's 208^3 grid: 0.295 ms a launch without, 0.267 ms with 64-256 rows; the bandwidth-bound
// instances and the forward pair kernel run slower with it)
constexpr int kDefaultSchemeAPrefetchRows = 128;

struct SourceState
{
    lbm_source s;
    std::vector<double> table;
};

template <typename T>
T* dalloc(size_t n, cudaError_t& err)
{
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, n * sizeof(T));
    return (T*)p;
}

}  // namespace

struct lbm_handle
{
    lbm_config cfg{};
    lbm_config lcfg{};                 // the grid this handle holds: cfg, or its z-slab (lbm_init)
    bool slab = false;
    int nz_global = 0;
    std::string err;
    int storage = LBM_STORE_F32;
    float scale = 1.0f;

    // geometry / mask
    HeightField geo;
    int stl_status = LBM_OK;
    std::vector<uint8_t> mask_override;
    int mo_dims[3] = {0, 0, 0};
    std::vector<double> blend_xy, field_xy;   // scheme A: caller's per-column fields (lbm_set_*_xy)

    std::vector<SourceState> srcs;
    std::vector<double> probe_xyz;

    // set-up results
    bool inited = false;
    int NXg = 0, NYg = 0, NZg = 0;
    double dt = 0.0;
    Layout L{};
    std::vector<uint8_t> mask;           // reference layout, halo-inclusive
    std::vector<int> probe_ijk;          // halo-inclusive cell coordinates, i = -1 unowned
    std::vector<int> probe_owned, probe_solid;

    // device state
    int device = 0;
    cudaStream_t stream = nullptr;
    void* f[2] = {nullptr, nullptr};   // population buffers (block-interleaved layout)
    int cur = 0;
    uint32_t* links = nullptr;
    uint32_t* near = nullptr;
    float* sig = nullptr;              // sig_x | sig_y | sig_z
    XFace xf{nullptr, nullptr};        // x-face exports and ghosts
    StepArgs sa{};
    GhostArgs ga{};
    Control* ctl = nullptr;            // device
    Control* ctl_host = nullptr;       // pinned staging
    SourceEntry* d_table = nullptr;
    SourceEntry* h_table = nullptr;    // pinned
    long long table_base = 0, table_rows = 0;
    int* d_probe_ijk = nullptr;
    double* d_probe_out = nullptr;
    double* h_probe_out = nullptr;     // pinned
    double* d_energy = nullptr;
    long long probe_pending = 0;        // rows recorded on the device, not yet on the host
    std::vector<double> series;
    bool halo_dirty = false;
    std::vector<float> rho0;             // scheme A: the initial density deviation lbm_set_density set

    long long step = 0;                // completed time steps
    long launches = 0;
    long h2d_bytes = 0, d2h_bytes = 0;

    // graphs: two full steps starting from buffer 0
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;

    // scheme A (family 01-04): omega and source-weight profiles, x-face arrays of both parities
    SchemeAArgs aa{};
    float* a_prof = nullptr;           // om_x | om_y | om_z | fld_x | fld_y | fld_z
    float* xgh_par[2] = {nullptr, nullptr};
    bool scheme_a() const { return cfg.scheme == LBM_SCHEME_A; }

    // z-slab exchange between handles of one process: message buffers
    // [send to lower | send to upper | received from lower | received from upper]
    // and the events that order the two handles' streams (lbm_slab_exchange)
    void* slab_buf = nullptr;
    size_t slab_msg_bytes = 0;
    cudaEvent_t ev_packed = nullptr, ev_read = nullptr;
    // a second stream for the small kernels that run beside a step (the batched step's
    // probe record; in lbm_adjoint_grad also the source and the reverse pass's source terms)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    // adjoint workspace (checkpoints, stored moments, adjoint populations),
    // kept between lbm_adjoint_grad calls; lbm_adjoint_release frees it
    void* adj_ws = nullptr;
    size_t adj_ws_bytes = 0;

    // kernel timing
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
    double kernel_ms = 0.0;
    long kernel_launches = 0;

    ~lbm_handle() { release(); }

    int fail(int code, const std::string& msg)
    {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* where)
    {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? LBM_ERR_OUT_OF_MEMORY : LBM_ERR_CUDA;
    }

    void release()
    {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
        ev_used = 0;
        for (int b = 0; b < 2; ++b)
        {
            if (f[b]) cudaFree(f[b]);
            f[b] = nullptr;
        }
        cudaFree(links); links = nullptr;
        cudaFree(near); near = nullptr;
        cudaFree(sig); sig = nullptr;
        cudaFree(xf.xexp); xf.xexp = nullptr;
        cudaFree(xf.xgh); xf.xgh = nullptr;
        xgh_par[0] = xgh_par[1] = nullptr;
        cudaFree(a_prof); a_prof = nullptr;
        cudaFree(ctl); ctl = nullptr;
        cudaFree(d_table); d_table = nullptr;
        cudaFree(d_probe_ijk); d_probe_ijk = nullptr;
        cudaFree(d_probe_out); d_probe_out = nullptr;
        cudaFree(d_energy); d_energy = nullptr;
        if (ctl_host) cudaFreeHost(ctl_host);
        if (h_table) cudaFreeHost(h_table);
        if (h_probe_out) cudaFreeHost(h_probe_out);
        ctl_host = nullptr; h_table = nullptr; h_probe_out = nullptr;
        if (adj_ws) cudaFree(adj_ws);
        adj_ws = nullptr;
        if (slab_buf) cudaFree(slab_buf);
        slab_buf = nullptr;
        slab_msg_bytes = 0;
        if (ev_packed) cudaEventDestroy(ev_packed);
        if (ev_read) cudaEventDestroy(ev_read);
        ev_packed = ev_read = nullptr;
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        ev_fork = ev_join = nullptr;
        if (side) cudaStreamDestroy(side);
        side = nullptr;
        adj_ws_bytes = 0;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        inited = false;
    }

    int nprobe() const { return (int)probe_xyz.size() / 3; }
};

// ---------------------------------------------------------------- helpers

namespace {

// DroneSource::update (06:221-238).
void drone_position(const lbm_source& s, double t, double& cx, double& cy, double& cz)
{
    double dx = s.ex - s.sx, dy = s.ey - s.sy, dz = s.ez - s.sz;
    double dist_total = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (dist_total < 1e-12 || s.speed < 1e-12)
    {
        cx = s.sx; cy = s.sy; cz = s.sz;
        return;
    }
    double travel_time = dist_total / s.speed;
    double r = t / travel_time;
    if (r > 1.0) r = 1.0;
    cx = s.sx + r * dx;
    cy = s.sy + r * dy;
    cz = s.sz + r * dz;
}

// Source time function at time t (06:579-581 Gaussian, 08:543 sine, Ricker,
// per-step table).
double source_value(const SourceState& st, double t, double dt)
{
    const lbm_source& p = st.s;
    switch (p.waveform)
    {
    case LBM_WAVE_GAUSS:
        return p.amp * std::exp(-0.5 * std::pow((t - p.t0) / p.sigma_t, 2));
    case LBM_WAVE_SINE:
        return p.amp * std::sin(2.0 * kPi * p.freq * t);
    case LBM_WAVE_RICKER:
    {
        double a = kPi * p.freq * (t - p.t0);
        a = a * a;
        return p.amp * (1.0 - 2.0 * a) * std::exp(-a);
    }
    case LBM_WAVE_TABLE:
    {
        const long s = std::lround(t / dt);
        if (s < 0 || s >= (long)st.table.size()) return 0.0;
        return p.amp * st.table[(size_t)s];
    }
    default:
        return 0.0;
    }
}

SourceEntry source_entry(const SourceState& st, double t, double dt)
{
    SourceEntry e;
    const double val = source_value(st, t, dt);
    drone_position(st.s, t, e.cx, e.cy, e.cz);
    e.mass = val * dt * st.s.gain;   // numerator of A (06:631)
    e.wsum = 0.0;
    return e;
}

int validate(const lbm_config& c, std::string& why)
{
    if (!(c.dx > 0)) return why = "dx must be > 0", LBM_ERR_BAD_CONFIG;
    if (!(c.tau > 0.5)) return why = "tau must be > 0.5", LBM_ERR_BAD_CONFIG;
    if (!(c.c_phys > 0)) return why = "c_phys must be > 0", LBM_ERR_BAD_CONFIG;
    if (!(c.x_max > c.x_min && c.y_max > c.y_min && c.z_max > c.z_min))
        return why = "empty domain", LBM_ERR_BAD_CONFIG;
    for (int f = 0; f < 6; ++f)
        if (c.face_bc[f] < LBM_BC_NSCBC || c.face_bc[f] > LBM_BC_PERIODIC)
            return why = "face_bc out of range", LBM_ERR_BAD_CONFIG;
    if (c.scheme != LBM_SCHEME_B && c.scheme != LBM_SCHEME_A) return why = "unknown scheme", LBM_ERR_BAD_CONFIG;
    if (!(c.dt >= 0)) return why = "dt must be >= 0 (0: cs*dx/c_phys)", LBM_ERR_BAD_CONFIG;
    int ncopy = 0, nnscbc = 0;
    for (int f = 0; f < 6; ++f)
    {
        ncopy += c.face_bc[f] == LBM_BC_COPY;
        nnscbc += c.face_bc[f] == LBM_BC_NSCBC;
    }
    if (c.scheme == LBM_SCHEME_B && ncopy) return why = "LBM_BC_COPY needs scheme A", LBM_ERR_BAD_CONFIG;
    int nper = 0;
    for (int f = 0; f < 6; ++f) nper += c.face_bc[f] == LBM_BC_PERIODIC;
    if (nper && (c.scheme != LBM_SCHEME_A || nper != 2 || c.face_bc[LBM_FACE_ZLO] != LBM_BC_PERIODIC ||
                 c.face_bc[LBM_FACE_ZHI] != LBM_BC_PERIODIC))
        return why = "LBM_BC_PERIODIC is scheme A on both z faces", LBM_ERR_BAD_CONFIG;
    if (c.sponge_blend != 0 && c.sponge_blend != 1) return why = "sponge_blend must be 0 or 1", LBM_ERR_BAD_CONFIG;
    if (c.sponge_blend && c.scheme != LBM_SCHEME_A) return why = "sponge_blend needs scheme A", LBM_ERR_BAD_CONFIG;
    if (c.sponge_blend && c.tau_sponge_max > 0)
        return why = "sponge_blend replaces the tau ramp (tau_sponge_max <= 0)", LBM_ERR_BAD_CONFIG;
    if (c.slab_k0 < 0 || c.slab_nz < 0) return why = "slab_k0 and slab_nz must be >= 0", LBM_ERR_BAD_CONFIG;
    if (c.slab_nz > 0)
    {
        const int nzg = (int)((c.z_max - c.z_min) / c.dx + 0.5);
        if (c.slab_k0 + c.slab_nz > nzg) return why = "the z-slab reaches past the grid", LBM_ERR_BAD_CONFIG;
        if (c.scheme != LBM_SCHEME_B) return why = "z-slabs run scheme B", LBM_ERR_BAD_CONFIG;
    }
    if (c.scheme == LBM_SCHEME_A)
    {
        if (c.storage != LBM_STORE_F32) return why = "scheme A runs on FP32 storage", LBM_ERR_BAD_CONFIG;
        if (nnscbc) return why = "scheme A has no characteristic (NSCBC) faces", LBM_ERR_BAD_CONFIG;
        if (ncopy != 0 && ncopy != 6) return why = "zero-gradient (LBM_BC_COPY) halos on all six faces or none",
                                      LBM_ERR_BAD_CONFIG;
        if (c.tau_sponge_max > 0 && c.tau_sponge_max < c.tau)
            return why = "tau_sponge_max must be >= tau", LBM_ERR_BAD_CONFIG;
    }
    if (c.storage != LBM_STORE_F32 && c.storage != LBM_STORE_F16)
        return why = "storage must be LBM_STORE_F32 or LBM_STORE_F16", LBM_ERR_BAD_CONFIG;
    if (c.storage == LBM_STORE_F16 && !(c.f16_scale > 0)) return why = "f16_scale must be > 0", LBM_ERR_BAD_CONFIG;
    if (!(c.sponge_width >= 0)) return why = "sponge_width must be >= 0", LBM_ERR_BAD_CONFIG;
    return LBM_OK;
}

// Per-axis sponge strength at interior cell centres (init_domain 06:491-506).
// sigma(x,y,z) = S((w - d)/w)^2 with d the distance to the nearest sponge
// face is monotone in d, so the per-cell value equals the maximum of the
// per-axis values; the kernel takes that maximum.  Values <= 1e-12 are the
// reference's "no sponge" (06:961) and are stored as 0.
void sponge_axis(const lbm_config& c, int axis, int n, std::vector<float>& out)
{
    const double lo[3] = {c.x_min, c.y_min, c.z_min};
    const double hi[3] = {c.x_max, c.y_max, c.z_max};
    const unsigned sf = c.sponge_faces;
    const double w = c.sponge_width * c.dx;
    out.resize((size_t)n);
    for (int i = 1; i <= n; ++i)
    {
        const double x = lo[axis] + ((i - 1) + 0.5) * c.dx;
        double d = 1e30;
        if (sf & (1u << (2 * axis))) d = std::min(d, x - lo[axis]);
        if (sf & (1u << (2 * axis + 1))) d = std::min(d, hi[axis] - x);
        double s = 0.0;
        if (d < w)
        {
            const double r = (w - d) / w;
            s = c.sponge_strength * r * r;
        }
        out[(size_t)i - 1] = s > 1e-12 ? (float)s : 0.0f;
    }
}

// Periodic z (01:105-107): halo planes 0 and nz + 1 repeat planes nz and 1,
// for a built mask and for a caller's (lbm_set_mask).
void periodic_z_mask(const lbm_config& c, int nx, int ny, int nz, uint8_t* m)
{
    if (c.face_bc[LBM_FACE_ZLO] != LBM_BC_PERIODIC) return;
    const size_t plane = (size_t)(nx + 2) * (ny + 2);
    std::copy(m + (size_t)nz * plane, m + (size_t)(nz + 1) * plane, m);
    std::copy(m + plane, m + 2 * plane, m + (size_t)(nz + 1) * plane);
}

// The voxelised mask of init_domain (06:460-531) in the reference's
// halo-inclusive layout: SOLID below the ground height of the column unless
// above sky_z, then the halo rules x faces, y faces, z faces in that order
// (a WALL face is SOLID, every other face FLUID).  gH_given: ground heights
// of every column already cast (on the GPU, bit-identical), else cast here.
void build_mask(const lbm_config& c, const HeightField& geo, int nx, int ny, int nz, uint8_t* m,
                const double* gH_given = nullptr)
{
    const int nxt = nx + 2, nyt = ny + 2, nzt = nz + 2;
    std::vector<double> gH((size_t)nxt * nyt, -1e30);
    const bool geom = c.use_geometry != 0;
    if (geom && gH_given)
    {
        std::copy(gH_given, gH_given + gH.size(), gH.begin());
    }
    else if (geom)
    {
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
        for (int j = 0; j < nyt; ++j)
            for (int i = 0; i < nxt; ++i)
            {
                const double x = c.x_min + ((i - 1) + 0.5) * c.dx;
                const double y = c.y_min + ((j - 1) + 0.5) * c.dx;
                gH[(size_t)j * nxt + i] = geo.ground_height(x, y);
            }
    }
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nzt; ++k)
        for (int j = 0; j < nyt; ++j)
        {
            const double z = c.z_min + ((k - 1) + 0.5) * c.dx;
            for (int i = 0; i < nxt; ++i)
            {
                const size_t idx = (size_t)i + (size_t)j * nxt + (size_t)k * nxt * nyt;
                uint8_t v = geom ? (z < gH[(size_t)j * nxt + i] ? 1 : 0) : 0;
                if (z > c.sky_z) v = 0;
                m[idx] = v;
            }
        }
    const auto wall = [&](int f) { return (uint8_t)(c.face_bc[f] == LBM_BC_WALL ? 1 : 0); };
    for (int k = 0; k < nzt; ++k)
        for (int j = 0; j < nyt; ++j)
        {
            m[(size_t)0 + (size_t)j * nxt + (size_t)k * nxt * nyt] = wall(LBM_FACE_XLO);
            m[(size_t)(nx + 1) + (size_t)j * nxt + (size_t)k * nxt * nyt] = wall(LBM_FACE_XHI);
        }
    for (int k = 0; k < nzt; ++k)
        for (int i = 0; i < nxt; ++i)
        {
            m[(size_t)i + (size_t)k * nxt * nyt] = wall(LBM_FACE_YLO);
            m[(size_t)i + (size_t)(ny + 1) * nxt + (size_t)k * nxt * nyt] = wall(LBM_FACE_YHI);
        }
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxt; ++i)
        {
            // a cut of a z-slab keeps the geometry of the neighbour slab's layer
            if (c.face_bc[LBM_FACE_ZLO] != kBcCut) m[(size_t)i + (size_t)j * nxt] = wall(LBM_FACE_ZLO);
            if (c.face_bc[LBM_FACE_ZHI] != kBcCut)
                m[(size_t)i + (size_t)j * nxt + (size_t)(nz + 1) * nxt * nyt] = wall(LBM_FACE_ZHI);
        }
    periodic_z_mask(c, nx, ny, nz, m);
}

void grid_size(const lbm_config& c, int& nx, int& ny, int& nz)
{
    // 06:332-334
    nx = (int)((c.x_max - c.x_min) / c.dx + 0.5);
    ny = (int)((c.y_max - c.y_min) / c.dx + 0.5);
    nz = (int)((c.z_max - c.z_min) / c.dx + 0.5);
}

// NVTX range around an entry point or a phase, for profilers (ncu --nvtx,
// Nsight Systems); without an attached tool it costs a pointer test.
struct NvtxRange
{
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

#define CK(expr, where)                                   \
    do                                                    \
    {                                                     \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return h->cuda_fail(e_, where); \
    } while (0)

// Scheme-A profiles on the device: omega of the tau ramp per axis (a cell's
// omega is the minimum over its three axes, equal to 1 / tau(min distance)
// since tau grows toward the faces; 02:164-179, 03:148-160), the field
// source's weight factors per axis, halo-inclusive (02:181, 03:166-169), and
// the background equilibrium feq(1, u0) the state is stored relative to
// (03:162-163).
int upload_scheme_a_profiles(lbm_handle* h)
{
    const lbm_config& c = h->cfg;
    const Layout& L = h->L;
    const int n[3] = {L.nx, L.ny, L.nz};
    const unsigned sf = c.sponge_faces;
    const int w = (int)c.sponge_width;
    std::vector<float> prof;
    prof.reserve((size_t)3 * (L.nx + L.ny + L.nz) + 6);
    for (int a = 0; a < 3; ++a)
        for (int g = 0; g < n[a]; ++g)
        {
            int d = 1 << 30;
            if (sf & (1u << (2 * a))) d = std::min(d, g);
            if (sf & (1u << (2 * a + 1))) d = std::min(d, n[a] - 1 - g);
            double tau = c.tau;
            if (c.tau_sponge_max > 0 && d >= 0 && d < w)
            {
                const double r = (double)(w - d) / w;
                tau = c.tau + (c.tau_sponge_max - c.tau) * r * r;
            }
            prof.push_back((float)(1.0 / tau));
        }
    const lbm_source* fs = nullptr;
    int fsi = -1;
    for (size_t i = 0; i < h->srcs.size(); ++i)
        if (h->srcs[i].s.injection == LBM_INJECT_FIELD)
        {
            fs = &h->srcs[i].s;
            fsi = (int)i;
        }
    const double lo[3] = {c.x_min, c.y_min, c.z_min};
    for (int a = 0; a < 3; ++a)
        for (int g = 0; g <= n[a] + 1; ++g)
        {
            double v = 1.0;
            if (fs)
            {
                const double sig = fs->sigma_cells * c.dx;
                const double ctr[3] = {fs->sx, fs->sy, fs->sz};
                const double x = lo[a] + ((g - 1) + 0.5) * c.dx - ctr[a];
                v = std::exp(-x * x / (2.0 * sig * sig));
            }
            prof.push_back((float)v);
        }
    // 01's blend strength per axis (01:207-225): depth th - dist into the
    // layer of thickness th = sponge_width dx, strength (depth / th)^2; the
    // cell's value (01's largest depth over the axes) is the largest of the
    // three, and values <= 1e-6 are 01's "not in the sponge" (01:302).
    const double hi[3] = {c.x_max, c.y_max, c.z_max};
    const double th = c.sponge_width * c.dx;
    for (int a = 0; a < 3; ++a)
        for (int g = 0; g < n[a]; ++g)
        {
            double sgv = 0.0;
            if (c.sponge_blend)
            {
                const double x = lo[a] + (g + 0.5) * c.dx;
                double dist = 0.0;
                if ((sf & (1u << (2 * a))) && x < lo[a] + th) dist = (lo[a] + th) - x;
                else if ((sf & (1u << (2 * a + 1))) && x > hi[a] - th) dist = x - (hi[a] - th);
                if (dist > 0.0)
                {
                    const double r = dist / th;
                    sgv = c.sponge_strength * r * r;
                }
            }
            prof.push_back(sgv > 1e-6 ? (float)sgv : 0.0f);
        }
    // the caller's per-column fields
    if (!h->blend_xy.empty() && !c.sponge_blend)
        return h->fail(LBM_ERR_BAD_CONFIG, "lbm_set_blend_xy needs sponge_blend = 1");
    const size_t off_sg_xy = prof.size();
    for (double v : h->blend_xy) prof.push_back(v > 1e-6 ? (float)v : 0.0f);
    const size_t off_fld_xy = prof.size();
    for (double v : h->field_xy) prof.push_back((float)v);
    if (!h->a_prof) CK(cudaMalloc(&h->a_prof, prof.size() * sizeof(float)), "scheme A profiles");
    CK(cudaMemcpyAsync(h->a_prof, prof.data(), prof.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream),
       "scheme A profiles");
    CK(cudaStreamSynchronize(h->stream), "scheme A profiles");
    h->h2d_bytes += (long)(prof.size() * sizeof(float));
    SchemeAArgs& b = h->aa;
    b.om_x = h->a_prof;
    b.om_y = b.om_x + L.nx;
    b.om_z = b.om_y + L.ny;
    b.fld_x = b.om_z + L.nz;
    b.fld_y = b.fld_x + L.nx + 2;
    b.fld_z = b.fld_y + L.ny + 2;
    b.sg_x = b.fld_z + L.nz + 2;
    b.sg_y = b.sg_x + L.nx;
    b.sg_z = b.sg_y + L.ny;
    b.blend = c.sponge_blend ? 1 : 0;
    b.zper = c.face_bc[LBM_FACE_ZLO] == LBM_BC_PERIODIC ? 1 : 0;
    b.sg_xy = h->blend_xy.empty() ? nullptr : h->a_prof + off_sg_xy;
    b.fld_xy = h->field_xy.empty() ? nullptr : h->a_prof + off_fld_xy;
    b.nx_col = L.nx;
    b.ny_col = L.ny;
    b.om_bulk = (float)(1.0 / c.tau);
    b.field_mode = fs ? fs->field_mode : -1;
    // a pre-step source enters the step that computes its arrivals, one step
    // ahead: nothing carries a value at t = 0 into the initial state
    if (fs && fs->field_mode == LBM_FIELD_PRE && source_entry(h->srcs[(size_t)fsi], 0.0, h->dt).mass != 0.0)
        return h->fail(LBM_ERR_UNSUPPORTED, "a LBM_FIELD_PRE source must be 0 at t = 0");
    b.src_index = fsi;
    b.nsrc = (int)h->srcs.size();
    double u2 = 0.0;
    for (int a = 0; a < 3; ++a)
    {
        b.flow[a] = (float)c.flow[a];
        u2 += c.flow[a] * c.flow[a];
    }
    for (int q = 0; q < Q; ++q)
    {
        const double cu = ex(q) * c.flow[0] + ey(q) * c.flow[1] + ez(q) * c.flow[2];
        b.base[q] = (float)(wd(q) * (3.0 * cu + 4.5 * cu * cu - 1.5 * u2));
        b.cu0[q] = (float)cu;
        b.fq[q] = (float)(wd(q) * (1.0 + 3.0 * cu));
    }
    b.u0sq = (float)u2;
    b.copy = c.face_bc[LBM_FACE_XLO] == LBM_BC_COPY ? 1 : 0;
    b.table = h->d_table;
    b.ctl = h->ctl;
    // L2 prefetch distance of the scheme-A instance with per-column fields (04's), in rows
    // (NLOS_LBM_A_PREFETCH_ROWS, 0 = off)
    b.prefetch_rows = kDefaultSchemeAPrefetchRows;
    if (const char* v = std::getenv("NLOS_LBM_A_PREFETCH_ROWS")) b.prefetch_rows = std::max(0, std::atoi(v));
    return LBM_OK;
}

}  // namespace

// ---------------------------------------------------------------- defaults

extern "C" void lbm_config_default(lbm_config* c)
{
    std::memset(c, 0, sizeof *c);
    c->x_min = 0.0; c->x_max = 1650.0;   // 06:250-252
    c->y_min = 0.0; c->y_max = 1150.0;
    c->z_min = 0.0; c->z_max = 250.0;
    c->dx = 2.0;                         // 06:253
    c->c_phys = 340.0;                   // 06:198
    c->tau = 0.55;                       // 06:268
    c->use_geometry = 1;                 // 06:248
    for (int f = 0; f < 6; ++f) c->face_bc[f] = LBM_BC_NSCBC;
    c->face_bc[LBM_FACE_ZLO] = LBM_BC_WALL;   // ground (06:520-531)
    c->sponge_faces = (1u << LBM_FACE_XLO) | (1u << LBM_FACE_XHI) | (1u << LBM_FACE_YLO) | (1u << LBM_FACE_YHI) |
                      (1u << LBM_FACE_ZHI);   // 06:491-496
    c->sponge_width = 20.0;              // 06:455
    c->sponge_strength = 0.35;           // 06:456
    c->sky_z = 120.0;                    // 06:458
    c->storage = LBM_STORE_F32;
    c->f16_scale = 1.0;
    c->device = 0;
    c->use_graphs = 1;
    c->verbose = 0;
}

extern "C" void lbm_source_default(lbm_source* s)
{
    std::memset(s, 0, sizeof *s);
    s->waveform = LBM_WAVE_GAUSS;
    s->t0 = 0.05;          // 06:579
    s->sigma_t = 0.005;    // 06:580
    s->injection = LBM_INJECT_GAUSS;
    s->gain = 1.0;         // 06:583
    s->sigma_cells = 1.25; // 06:588
    s->radius = 2;         // 06:587
}

extern "C" const char* lbm_status_string(int s)
{
    switch (s)
    {
    case LBM_OK: return "ok";
    case LBM_WARN_STL_NOT_LOADED: return "warning: STL not loaded, using empty geometry";
    case LBM_WARN_PROBE_IN_SOLID: return "warning: probe inside a SOLID cell";
    case LBM_WARN_STL_TRUNCATED: return "warning: STL truncated, missing triangles read as zeros";
    case LBM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LBM_ERR_BAD_CONFIG: return "bad configuration";
    case LBM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case LBM_ERR_CUDA: return "CUDA error";
    case LBM_ERR_NAN: return "non-finite value in probe series";
    case LBM_ERR_STATE: return "call out of order";
    case LBM_ERR_CAPACITY: return "output buffer too small";
    case LBM_ERR_NO_DEVICE: return "no CUDA device";
    case LBM_ERR_IO: return "I/O error";
    case LBM_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

extern "C" const char* lbm_version(void) { return "nlos_lbm 0.1 (sm_100a)"; }

// ---------------------------------------------------------------- lifetime

extern "C" int lbm_create(const lbm_config* cfg, lbm_handle** out)
{
    if (!cfg || !out) return LBM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::string why;
    int st = validate(*cfg, why);
    if (st != LBM_OK) return st;
    auto* h = new (std::nothrow) lbm_handle();
    if (!h) return LBM_ERR_OUT_OF_MEMORY;
    h->cfg = *cfg;
    h->storage = cfg->storage;
    h->scale = cfg->storage == LBM_STORE_F16 ? (float)cfg->f16_scale : 1.0f;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
        delete h;
        return LBM_ERR_NO_DEVICE;
    }
    if (cfg->device < 0 || cfg->device >= ndev)
    {
        delete h;
        return LBM_ERR_BAD_CONFIG;
    }
    h->device = cfg->device;
    *out = h;
    return LBM_OK;
}

extern "C" int lbm_destroy(lbm_handle* h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    delete h;
    return LBM_OK;
}

extern "C" const char* lbm_last_error(lbm_handle* h) { return h ? h->err.c_str() : ""; }

// ---------------------------------------------------------------- geometry

extern "C" int lbm_set_geometry_stl(lbm_handle* h, const char* path, double scale, double sx, double sy, double sz)
{
    if (!h || !path) return LBM_ERR_INVALID_ARGUMENT;
    const int r = h->geo.load_stl(path, scale, sx, sy, sz);
    h->stl_status = r == HeightField::kStlLoaded ? LBM_OK
                  : r == HeightField::kStlNotOpened ? LBM_WARN_STL_NOT_LOADED
                                                    : LBM_WARN_STL_TRUNCATED;
    if (r == HeightField::kStlNotOpened) h->err = std::string("STL not loaded: ") + path;
    if (r == HeightField::kStlTruncated)
        h->err = std::string("STL ends before the triangle count of its header; missing records read as zeros: ") +
                 path;
    return h->stl_status;
}

extern "C" int lbm_set_geometry_triangles(lbm_handle* h, const float* tris, int ntris, double scale, double sx,
                                          double sy, double sz)
{
    if (!h || ntris < 0 || (ntris > 0 && !tris)) return LBM_ERR_INVALID_ARGUMENT;
    h->geo.set_triangles(tris, ntris, scale, sx, sy, sz);
    h->stl_status = LBM_OK;
    return LBM_OK;
}

namespace {
int set_columns(lbm_handle* h, const double* v, long count, std::vector<double>& out, const char* what)
{
    if (!h || !v) return LBM_ERR_INVALID_ARGUMENT;
    if (h->inited) return h->fail(LBM_ERR_STATE, "per-column fields are set before lbm_init");
    if (h->cfg.scheme != LBM_SCHEME_A) return h->fail(LBM_ERR_UNSUPPORTED, "per-column fields are scheme A");
    int nx = 0, ny = 0, nz = 0;
    grid_size(h->cfg, nx, ny, nz);
    if (count != (long)nx * ny) return h->fail(LBM_ERR_INVALID_ARGUMENT, what);
    out.assign(v, v + count);
    return LBM_OK;
}
}  // namespace

extern "C" int lbm_set_blend_xy(lbm_handle* h, const double* s_xy, long count)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    return set_columns(h, s_xy, count, h->blend_xy, "blend field size mismatch");
}

extern "C" int lbm_set_field_weights_xy(lbm_handle* h, const double* w_xy, long count)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    return set_columns(h, w_xy, count, h->field_xy, "weight field size mismatch");
}

extern "C" int lbm_set_mask(lbm_handle* h, const uint8_t* mask, int nx_t, int ny_t, int nz_t)
{
    if (!h || !mask || nx_t < 3 || ny_t < 3 || nz_t < 3) return LBM_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)nx_t * ny_t * nz_t;
    h->mask_override.assign(mask, mask + n);
    for (auto& m : h->mask_override) m = m ? 1 : 0;
    h->mo_dims[0] = nx_t; h->mo_dims[1] = ny_t; h->mo_dims[2] = nz_t;
    return LBM_OK;
}

// ---------------------------------------------------------------- sources / probes

extern "C" int lbm_add_source(lbm_handle* h, const lbm_source* s)
{
    if (!h || !s) return LBM_ERR_INVALID_ARGUMENT;
    if ((int)h->srcs.size() >= kMaxSources) return h->fail(LBM_ERR_UNSUPPORTED, "at most 8 sources");
    if (s->injection == LBM_INJECT_GAUSS && (s->radius < 0 || s->radius > 3 || !(s->sigma_cells > 0)))
        return h->fail(LBM_ERR_INVALID_ARGUMENT, "Gaussian stencil needs radius 0..3 and sigma_cells > 0");
    if (s->injection != LBM_INJECT_GAUSS && s->injection != LBM_INJECT_TRILINEAR && s->injection != LBM_INJECT_FIELD)
        return h->fail(LBM_ERR_INVALID_ARGUMENT, "unknown injection");
    if (h->cfg.scheme == LBM_SCHEME_A)
    {
        if (s->injection != LBM_INJECT_FIELD)
            return h->fail(LBM_ERR_UNSUPPORTED, "scheme A takes field sources (LBM_INJECT_FIELD) only");
        if (!h->srcs.empty()) return h->fail(LBM_ERR_UNSUPPORTED, "scheme A takes one field source");
        if (!(s->sigma_cells > 0)) return h->fail(LBM_ERR_INVALID_ARGUMENT, "field source needs sigma_cells > 0");
        if (s->field_mode != LBM_FIELD_DST && s->field_mode != LBM_FIELD_FORCE && s->field_mode != LBM_FIELD_PRE)
            return h->fail(LBM_ERR_INVALID_ARGUMENT, "unknown field_mode");
    }
    else if (s->injection == LBM_INJECT_FIELD)
    {
        return h->fail(LBM_ERR_UNSUPPORTED, "field sources need scheme A");
    }
    if (s->waveform < LBM_WAVE_GAUSS || s->waveform > LBM_WAVE_TABLE)
        return h->fail(LBM_ERR_INVALID_ARGUMENT, "unknown waveform");
    if (s->waveform == LBM_WAVE_TABLE && (s->table_len < 0 || (s->table_len > 0 && !s->table)))
        return h->fail(LBM_ERR_INVALID_ARGUMENT, "table waveform needs table samples");
    SourceState st;
    st.s = *s;
    if (s->waveform == LBM_WAVE_TABLE) st.table.assign(s->table, s->table + s->table_len);
    st.s.table = nullptr;
    h->srcs.push_back(std::move(st));
    h->table_rows = 0;   // schedule must be rebuilt
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    if (h->inited && h->scheme_a()) return upload_scheme_a_profiles(h);
    return LBM_OK;
}

extern "C" int lbm_clear_sources(lbm_handle* h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    h->srcs.clear();
    h->table_rows = 0;
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    if (h->inited && h->scheme_a()) return upload_scheme_a_profiles(h);
    return LBM_OK;
}

extern "C" int lbm_set_probes(lbm_handle* h, const double* xyz, int n)
{
    if (!h || n < 0 || (n > 0 && !xyz)) return LBM_ERR_INVALID_ARGUMENT;
    if (h->inited) return h->fail(LBM_ERR_STATE, "probes are fixed at lbm_init");
    h->probe_xyz.assign(xyz, xyz + 3 * (size_t)n);
    return LBM_OK;
}

extern "C" int lbm_probe_info(lbm_handle* h, int* owned, int* in_solid)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    if (!h->inited) return LBM_ERR_STATE;
    for (int p = 0; p < h->nprobe(); ++p)
    {
        if (owned) owned[p] = h->probe_owned[p];
        if (in_solid) in_solid[p] = h->probe_solid[p];
    }
    return LBM_OK;
}

// ---------------------------------------------------------------- init

extern "C" int lbm_init(lbm_handle* h)
{
    NvtxRange range("lbm_init");
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    h->release();
    CK(cudaSetDevice(h->device), "cudaSetDevice");

    // The grid this handle holds: the whole configured grid, or its z-slab
    // (layers slab_k0 .. slab_k0 + slab_nz - 1) with the cut faces marked.
    {
        int gx, gy, gz;
        grid_size(h->cfg, gx, gy, gz);
        h->nz_global = gz;
        h->lcfg = h->cfg;
        h->slab = h->cfg.slab_nz > 0;
        if (h->slab)
        {
            lbm_config& l = h->lcfg;
            l.z_min = h->cfg.z_min + h->cfg.slab_k0 * h->cfg.dx;
            l.z_max = l.z_min + h->cfg.slab_nz * h->cfg.dx;
            if (h->cfg.slab_k0 > 0) l.face_bc[LBM_FACE_ZLO] = kBcCut;
            if (h->cfg.slab_k0 + h->cfg.slab_nz < gz) l.face_bc[LBM_FACE_ZHI] = kBcCut;
        }
    }
    const lbm_config& c = h->lcfg;

    // Grid (06:330-334, MPI size 1: one block, off = 0) and time step (06:200-203).
    grid_size(c, h->NXg, h->NYg, h->NZg);
    h->dt = (kCs * c.dx) / c.c_phys;
    if (c.dt > 0) h->dt = c.dt;
    const int nx = h->NXg, ny = h->NYg, nz = h->NZg;
    if (nx < 1 || ny < 1 || nz < 1) return h->fail(LBM_ERR_BAD_CONFIG, "grid has no cells");
    const int nxt = nx + 2, nyt = ny + 2, nzt = nz + 2;
    const size_t nloc = (size_t)nxt * nyt * nzt;

    Layout& L = h->L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.pitch = (nx + 2 + 31) / 32 * 32;
    L.words_per_row = (L.pitch / 32 + 1) & ~1;   // even: a block's two words load as one 8-byte word
    L.plane = (long long)L.pitch * nyt;
    L.bc = block_cells(h->storage == LBM_STORE_F16 ? 2 : 4);
    L.bc_shift = L.bc == 64 ? 6 : 5;
    L.nb = (nx + L.bc - 1) / L.bc;
    L.row_stride = (long long)L.nb * Q * L.bc;
    L.plane_stride = L.row_stride * nyt;
    L.total = kFrontElems + L.plane_stride * nzt + kBackElems;

    // The two population buffers and the links words must fit in the free
    // device memory: a grid that cannot fit fails here, before any host or
    // device allocation (later allocations still report their own failure).
    {
        const double need = 2.0 * (double)L.total * (h->storage == LBM_STORE_F16 ? 2 : 4) + 4.0 * (double)L.plane * nzt;
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        if (need > (double)free_b)
        {
            char msg[160];
            std::snprintf(msg, sizeof msg, "the grid needs at least %.1f GB of device memory, %.1f GB free", need / 1e9,
                          (double)free_b / 1e9);
            return h->fail(LBM_ERR_OUT_OF_MEMORY, msg);
        }
    }

    // Mask (init_domain 06:453-532).
    if (!h->mask_override.empty())
    {
        if (h->mo_dims[0] != nxt || h->mo_dims[1] != nyt || h->mo_dims[2] != nzt)
            return h->fail(LBM_ERR_INVALID_ARGUMENT, "lbm_set_mask dimensions do not match the grid");
        h->mask = h->mask_override;
        periodic_z_mask(c, nx, ny, nz, h->mask.data());
    }
    else
    {
        try
        {
            h->mask.assign(nloc, 0);
        }
        catch (const std::bad_alloc&)
        {
            return h->fail(LBM_ERR_OUT_OF_MEMORY, "host mask");
        }
        // the ray cast of every column runs on the GPU (voxel.cu) when there is geometry
        std::vector<double> gH;
        if (c.use_geometry && h->geo.triangle_count() > 0)
        {
            gH.assign((size_t)nxt * nyt, 0.0);
            CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            const int ve = ground_height_device(h->geo, c.x_min, c.y_min, c.dx, nxt, nyt, gH.data(), h->stream);
            if (ve != 0) return h->cuda_fail((cudaError_t)ve, "ground heights");
            h->launches += 1;
        }
        build_mask(c, h->geo, nx, ny, nz, h->mask.data(), gH.empty() ? nullptr : gH.data());
    }

    // Sponge profiles.
    std::vector<float> sx, sy, sz;
    sponge_axis(c, 0, nx, sx);
    sponge_axis(c, 1, ny, sy);
    if (!h->slab)
    {
        sponge_axis(c, 2, nz, sz);
    }
    else
    {
        // distances to the faces of the whole grid, sliced to this slab
        std::vector<float> szg;
        sponge_axis(h->cfg, 2, h->nz_global, szg);
        sz.assign(szg.begin() + h->cfg.slab_k0, szg.begin() + h->cfg.slab_k0 + nz);
    }

    // Device buffers.
    if (!h->stream) CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!h->side)
    {
        CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking), "side stream");
        CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming), "side stream events");
        CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming), "side stream events");
    }
    const size_t esz = h->storage == LBM_STORE_F16 ? 2 : 4;
    const size_t pop_bytes = (size_t)L.total * esz;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2; ++b)
    {
        if (e == cudaSuccess) e = cudaMalloc(&h->f[b], pop_bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->f[b], 0, pop_bytes, h->stream);   // g = 0: rest state (06:388-395)
    }
    const size_t cells = (size_t)L.plane * nzt;
    h->links = dalloc<uint32_t>(cells, e);
    const size_t near_words = (size_t)nzt * nyt * L.words_per_row;
    h->near = dalloc<uint32_t>(near_words, e);
    // sig_x padded with zeros to whole 64-cell blocks (the FP16 step loads a pair per lane unguarded)
    const int nxs = (nx + 63) / 64 * 64;
    h->sig = dalloc<float>((size_t)nxs + ny + nz, e);
    const size_t n_xexp = (size_t)2 * Q * ny * nz, n_xgh = (size_t)2 * Q * nyt * nzt;
    h->xf.xexp = dalloc<float>(n_xexp, e);
    const size_t n_xgh_all = n_xgh * (h->scheme_a() ? 2 : 1);   // scheme A: one array per step parity
    h->xf.xgh = dalloc<float>(n_xgh_all, e);
    h->ctl = dalloc<Control>(1, e);
    if (e != cudaSuccess) return h->cuda_fail(e, "device allocation");
    CK(cudaMemsetAsync(h->ctl, 0, sizeof(Control), h->stream), "memset control");
    CK(cudaMemsetAsync(h->links, 0, cells * sizeof(uint32_t), h->stream), "memset links");
    CK(cudaMemsetAsync(h->near, 0, near_words * sizeof(uint32_t), h->stream), "memset near");
    CK(cudaMemsetAsync(h->xf.xexp, 0, n_xexp * sizeof(float), h->stream), "memset x faces");
    CK(cudaMemsetAsync(h->xf.xgh, 0, n_xgh_all * sizeof(float), h->stream), "memset x faces");
    h->xgh_par[0] = h->xf.xgh;
    h->xgh_par[1] = h->xf.xgh + (h->scheme_a() ? n_xgh : 0);
    CK(cudaMallocHost(&h->ctl_host, sizeof(Control)), "cudaMallocHost");
    *h->ctl_host = Control{};
    CK(cudaMemsetAsync(h->sig, 0, (size_t)nxs * 4, h->stream), "memset sponge");
    CK(cudaMemcpyAsync(h->sig, sx.data(), sx.size() * 4, cudaMemcpyHostToDevice, h->stream), "upload sponge");
    CK(cudaMemcpyAsync(h->sig + nxs, sy.data(), sy.size() * 4, cudaMemcpyHostToDevice, h->stream), "upload sponge");
    CK(cudaMemcpyAsync(h->sig + nxs + ny, sz.data(), sz.size() * 4, cudaMemcpyHostToDevice, h->stream),
       "upload sponge");
    {
        uint8_t* d_mask = nullptr;
        CK(cudaMalloc(&d_mask, nloc), "mask upload buffer");
        e = cudaMemcpyAsync(d_mask, h->mask.data(), nloc, cudaMemcpyHostToDevice, h->stream);
        // links[c] belongs to the cell with linear index c (interior cells only)
        if (e == cudaSuccess) e = launch_build_links(d_mask, h->links, h->near, L, h->stream);
        if (e == cudaSuccess && h->scheme_a())
        {
            const int ps = upload_scheme_a_profiles(h);
            if (ps != LBM_OK)
            {
                cudaFree(d_mask);
                return ps;
            }
            e = launch_init_a((float*)h->f[0], (float*)h->f[1], h->xgh_par[0], h->xgh_par[1], d_mask, L, h->aa,
                              h->stream);
            h->launches += 1;
            if (e == cudaSuccess && h->aa.zper)
            {
                StepArgs sa = h->sa;
                sa.links = h->links;
                for (int p = 0; p < 2 && e == cudaSuccess; ++p) e = launch_zper_a((float*)h->f[p], L, sa, h->stream);
                h->launches += 2;
            }
        }
        cudaError_t e2 = cudaStreamSynchronize(h->stream);
        cudaFree(d_mask);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess) return h->cuda_fail(e, "build links");
        h->launches += 1;
    }

    h->sa.links = h->links;
    h->sa.near = h->near;
    h->sa.sig_x = h->sig;
    h->sa.sig_y = h->sig + (nx + 63) / 64 * 64;
    h->sa.sig_z = h->sa.sig_y + ny;
    h->sa.omega = (float)(1.0 / c.tau);
    h->sa.xf = h->xf;
    {
        const cudaError_t e = prepare_step(h->storage == LBM_STORE_F16 ? 1 : 0);
        if (e != cudaSuccess) return h->cuda_fail(e, "step set-up");
    }

    // Open faces for the ghost kernel.
    h->ga = GhostArgs{};
    h->ga.scale = h->scale;
    h->ga.xf = h->xf;
    long long first = 0;
    for (int f = 0; f < 6; ++f)
    {
        if (c.face_bc[f] != LBM_BC_NSCBC) continue;
        GhostFace gf;
        gf.axis = f / 2;
        gf.side = f % 2;
        gf.nu = gf.axis == 0 ? ny : nx;
        gf.nv = gf.axis == 2 ? ny : nz;
        gf.first = first;
        // the ghost kernels index within a face in 32 bits
        if ((long long)gf.nu * gf.nv > 0x7fffffffLL) return h->fail(LBM_ERR_UNSUPPORTED, "an open face of 2^31 cells or more");
        first += (long long)gf.nu * gf.nv;
        h->ga.face[h->ga.nfaces++] = gf;
    }
    h->ga.total = first;

    // Probes (06:415-437).
    int status = h->stl_status;
    const int np = h->nprobe();
    h->probe_ijk.assign((size_t)np * 3, -1);
    h->probe_owned.assign((size_t)np, 0);
    h->probe_solid.assign((size_t)np, 0);
    for (int p = 0; p < np; ++p)
    {
        const int gi = (int)std::floor((h->probe_xyz[3 * p] - c.x_min) / c.dx);
        const int gj = (int)std::floor((h->probe_xyz[3 * p + 1] - c.y_min) / c.dx);
        const int gk = (int)std::floor((h->probe_xyz[3 * p + 2] - c.z_min) / c.dx);
        if (gi >= 0 && gi < nx && gj >= 0 && gj < ny && gk >= 0 && gk < nz)
        {
            h->probe_owned[p] = 1;
            h->probe_ijk[3 * p] = gi + 1;
            h->probe_ijk[3 * p + 1] = gj + 1;
            h->probe_ijk[3 * p + 2] = gk + 1;
            const size_t idx = (size_t)(gi + 1) + (size_t)(gj + 1) * nxt + (size_t)(gk + 1) * nxt * nyt;
            if (h->mask[idx])
            {
                h->probe_solid[p] = 1;
                if (status == LBM_OK) status = LBM_WARN_PROBE_IN_SOLID;
                if (c.verbose) std::printf("WARNING: Probe %d is trapped inside SOLID building!\n", p);
            }
        }
    }
    const int npa = std::max(np, 1);
    h->d_probe_ijk = dalloc<int>((size_t)npa * 3, e);
    h->d_probe_out = dalloc<double>((size_t)npa * kProbeRows, e);
    h->d_energy = dalloc<double>((size_t)npa, e);
    if (e != cudaSuccess) return h->cuda_fail(e, "probe buffers");
    CK(cudaMallocHost(&h->h_probe_out, (size_t)npa * kProbeRows * sizeof(double)), "cudaMallocHost");
    if (np)
        CK(cudaMemcpyAsync(h->d_probe_ijk, h->probe_ijk.data(), (size_t)np * 3 * sizeof(int), cudaMemcpyHostToDevice,
                           h->stream),
           "upload probes");
    CK(cudaMemsetAsync(h->d_energy, 0, (size_t)npa * 8, h->stream), "memset energy");

    // Source schedule buffers (sized for the maximum source count so sources
    // may change after init).
    const size_t ns = kMaxSources;
    h->d_table = dalloc<SourceEntry>(ns * (kTableRows + 1), e);   // + 1: scheme-A forcing reads row s + 1
    if (e != cudaSuccess) return h->cuda_fail(e, "source table");
    CK(cudaMallocHost(&h->h_table, ns * (kTableRows + 1) * sizeof(SourceEntry)), "cudaMallocHost");
    h->table_base = 0;
    h->table_rows = 0;

    h->series.clear();
    h->probe_pending = 0;
    h->step = 0;
    h->cur = 0;
    h->halo_dirty = false;
    CK(cudaStreamSynchronize(h->stream), "init sync");
    h->h2d_bytes = h->d2h_bytes = 0;
    h->inited = true;
    if (c.verbose)
        std::printf("Grid: %d x %d x %d  (dx=%g m)\ndt=%g s\n", nx, ny, nz, c.dx, h->dt);
    return status;
}

// ---------------------------------------------------------------- stepping internals

namespace {

SourceArgs source_args(lbm_handle* h, bool batched)
{
    SourceArgs a{};
    a.nsrc = (int)h->srcs.size();
    for (int s = 0; s < a.nsrc; ++s)
    {
        const lbm_source& p = h->srcs[s].s;
        a.st[s].injection = p.injection;
        a.st[s].radius = p.radius;
        a.st[s].sigma2 = (p.sigma_cells * h->cfg.dx) * (p.sigma_cells * h->cfg.dx);   // 06:589
    }
    a.table = batched ? h->d_table : nullptr;
    a.ctl = batched ? h->ctl : nullptr;
    a.x_min = h->cfg.x_min;
    a.y_min = h->cfg.y_min;
    a.z_min = h->cfg.z_min;    // the whole grid's origin: weights as in an undivided run
    a.k_off = h->slab ? h->cfg.slab_k0 : 0;
    a.dx = h->cfg.dx;
    a.scale = h->scale;
    return a;
}

ProbeArgs probe_args(lbm_handle* h, bool batched, long long direct_row)
{
    ProbeArgs a{};
    a.n = h->nprobe();
    a.ijk = h->d_probe_ijk;
    a.out = h->d_probe_out;
    a.energy = h->d_energy;
    a.ctl = batched ? h->ctl : nullptr;
    a.direct_row = direct_row;
    a.scale = h->scale;
    a.nonfinite = &h->ctl->nonfinite;
    return a;
}

// Arguments of the scheme-A kernels of step s, which reads buffer `parity`:
// batched steps read the source schedule from the device table, direct
// calls get the masses of steps s and s + 1 from the host.
void scheme_a_args(lbm_handle* h, int parity, bool batched, long long s, StepArgs& sa, SchemeAArgs& b)
{
    sa = h->sa;
    sa.xf.xgh = h->xgh_par[parity];
    b = h->aa;
    b.table = h->d_table;
    b.ctl = batched ? h->ctl : nullptr;
    b.xgh_out = h->xgh_par[parity ^ 1];
    b.mass_direct[0] = b.mass_direct[1] = 0.f;
    if (!batched && b.field_mode >= 0)
    {
        const SourceState& fs = h->srcs[(size_t)b.src_index];
        b.mass_direct[0] = (float)source_entry(fs, (double)s * h->dt, h->dt).mass;
        b.mass_direct[1] = (float)source_entry(fs, (double)(s + 1) * h->dt, h->dt).mass;
    }
}

// The fused step of the handle's scheme from buffer `parity` into the other,
// bracketed by timing events when kernel timing is on.
cudaError_t timed_step_launch(lbm_handle* h, int parity, bool batched, long long s)
{
    const auto launch = [&]() {
        if (!h->scheme_a())
            return launch_step(h->storage, h->f[parity], h->f[parity ^ 1], h->L, h->sa, h->scale,
                               h->stream);
        StepArgs sa;
        SchemeAArgs b;
        scheme_a_args(h, parity, batched, s, sa, b);
        return launch_step_a((const float*)h->f[parity], (float*)h->f[parity ^ 1], h->L, sa, b, h->stream);
    };
    cudaError_t e;
    if (h->timing)
    {
        if (h->ev_used + 2 > h->ev.size())
        {
            for (int n = 0; n < 64; ++n)
            {
                cudaEvent_t x;
                e = cudaEventCreate(&x);
                if (e != cudaSuccess) return e;
                h->ev.push_back(x);
            }
        }
        e = cudaEventRecord(h->ev[h->ev_used], h->stream);
        if (e != cudaSuccess) return e;
        e = launch();
        if (e != cudaSuccess) return e;
        e = cudaEventRecord(h->ev[h->ev_used + 1], h->stream);
        h->ev_used += 2;
        return e;
    }
    return launch();
}

// Collect the kernel times recorded since the last harvest (synchronises).
int harvest_timing(lbm_handle* h)
{
    if (!h->timing || h->ev_used == 0) return LBM_OK;
    cudaError_t e = cudaEventSynchronize(h->ev[h->ev_used - 1]);
    if (e != cudaSuccess) return h->cuda_fail(e, "timing");
    for (size_t n = 0; n < h->ev_used; n += 2)
    {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, h->ev[n], h->ev[n + 1]);
        if (e != cudaSuccess) return h->cuda_fail(e, "timing");
        h->kernel_ms += ms;
        h->kernel_launches += 1;
    }
    h->ev_used = 0;
    return LBM_OK;
}

// One full time step on the device (source -> ghosts -> fused step ->
// probes), reading the step index from the device control block.
cudaError_t enqueue_batched_step(lbm_handle* h, int parity, int& kernels, bool captured = false)
{
    cudaError_t e = cudaSuccess;
    void* fc = h->f[parity];
    void* fn = h->f[parity ^ 1];
    kernels = 0;
    if (h->scheme_a())
    {
        // the field source acts inside the step; halo copies and probes read the same buffer
        StepArgs sa;
        SchemeAArgs b;
        scheme_a_args(h, parity, true, 0, sa, b);
        e = timed_step_launch(h, parity, true, 0);
        if (e != cudaSuccess) return e;
        kernels++;
        if (b.copy)
        {
            e = launch_copy_a((const float*)fc, (float*)fn, h->L, sa, b, h->stream);
            if (e != cudaSuccess) return e;
            kernels++;
        }
        e = launch_probe_a((const float*)fc, h->L, sa, b, probe_args(h, true, 0), h->stream);
        kernels++;
        return e;
    }
    if (!h->srcs.empty())
    {
        e = launch_source(h->storage, fc, h->L, h->sa, source_args(h, true), h->stream);
        if (e != cudaSuccess) return e;
        kernels++;
    }
    if (h->ga.total > 0)
    {
        e = launch_ghost(h->storage, fc, h->L, h->ga, h->stream);
        if (e != cudaSuccess) return e;
        kernels++;
    }
    if (!captured)
    {
        e = timed_step_launch(h, parity, true, 0);
        if (e != cudaSuccess) return e;
        kernels++;
        e = launch_probe(h->storage, fc, h->L, h->sa, probe_args(h, true, 0), h->stream);
        kernels++;
        return e;
    }
    // In the captured graph the probe record, which reads this step's input
    // buffer and ghosts (the step only reads them) and advances the device step
    // counter (no scheme-B step kernel reads it), is a branch beside the step,
    // joined before the next step's source reads the counter.  Direct launches
    // of single steps keep one stream (no graph amortises the fork and join).
    e = cudaEventRecord(h->ev_fork, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
    if (e == cudaSuccess) e = launch_probe(h->storage, fc, h->L, h->sa, probe_args(h, true, 0), h->side);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev_join, h->side);
    if (e != cudaSuccess) return e;
    kernels++;
    e = timed_step_launch(h, parity, true, 0);
    if (e != cudaSuccess) return e;
    kernels++;
    return cudaStreamWaitEvent(h->stream, h->ev_join, 0);
}

int build_graph(lbm_handle* h)
{
    if (h->graph) return LBM_OK;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return h->cuda_fail(e, "begin capture");
    int k0 = 0, k1 = 0;
    cudaError_t le = enqueue_batched_step(h, 0, k0, true);
    if (le == cudaSuccess) le = enqueue_batched_step(h, 1, k1, true);
    e = cudaStreamEndCapture(h->stream, &g);
    if (le != cudaSuccess) e = le;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&h->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess)
    {
        h->graph = nullptr;
        return h->cuda_fail(e, "graph capture");
    }
    h->graph_kernels = k0 + k1;
    return LBM_OK;
}

// Moves the probe rows buffered on the device to the host series.
int drain_probes(lbm_handle* h)
{
    const int np = h->nprobe();
    if (np == 0 || h->probe_pending == 0) return LBM_OK;
    const size_t n = (size_t)h->probe_pending * np;
    CK(cudaMemcpyAsync(h->h_probe_out, h->d_probe_out, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
       "probe download");
    h->d2h_bytes += (long)(n * sizeof(double));
    CK(cudaStreamSynchronize(h->stream), "probe download");
    h->series.insert(h->series.end(), h->h_probe_out, h->h_probe_out + n);
    h->probe_pending = 0;
    for (size_t i = 0; i < n; ++i)
        if (h->probe_owned[i % np] && !std::isfinite(h->h_probe_out[i]))
            return h->fail(LBM_ERR_NAN, "non-finite probe value");
    return LBM_OK;
}

// Source entry of step time t for this handle.  A z-slab whose source
// stencil reaches past its own layers gets the fluid-weight sum of the whole
// stencil (k_source divides by it), from the geometry: the mask of any cell
// of the whole grid follows from the ground heights (06:469-489); with a
// caller's mask (lbm_set_mask) cells beyond the slab's halo count as fluid.
SourceEntry entry_for(const lbm_handle* h, const SourceState& st, double t)
{
    SourceEntry e = source_entry(st, t, h->dt);
    if (!h->slab || e.mass == 0.0) return e;
    const lbm_config& c = h->cfg;
    const lbm_source& p = st.s;
    const int k0 = c.slab_k0, k1 = c.slab_k0 + c.slab_nz, nzg = h->nz_global;
    const int nx = h->NXg, ny = h->NYg;
    const auto fluid = [&](int gi, int gj, int gk) {
        if (gi < 0 || gi >= nx || gj < 0 || gj >= ny || gk < 0 || gk >= nzg) return false;
        if (!h->mask_override.empty())
        {
            if (gk < k0 - 1 || gk > k1) return true;
            const size_t nxt = nx + 2, nyt = ny + 2;
            return h->mask[(size_t)(gi + 1) + (size_t)(gj + 1) * nxt + (size_t)(gk - k0 + 1) * nxt * nyt] == 0;
        }
        if (!c.use_geometry) return true;
        const double x = c.x_min + (gi + 0.5) * c.dx, y = c.y_min + (gj + 0.5) * c.dx, z = c.z_min + (gk + 0.5) * c.dx;
        if (z > c.sky_z) return true;
        return !(z < h->geo.ground_height(x, y));
    };
    std::vector<int> cells;   // gi, gj, gk
    std::vector<double> w;
    if (p.injection == LBM_INJECT_TRILINEAR)
    {
        const double fx = (e.cx - c.x_min) / c.dx - 0.5, fy = (e.cy - c.y_min) / c.dx - 0.5,
                     fz = (e.cz - c.z_min) / c.dx - 0.5;
        const int i0 = (int)std::floor(fx), j0 = (int)std::floor(fy), kk0 = (int)std::floor(fz);
        const double tx = fx - i0, ty = fy - j0, tz = fz - kk0;
        for (int b = 0; b < 8; ++b)
        {
            cells.insert(cells.end(), {i0 + (b & 1), j0 + ((b >> 1) & 1), kk0 + (b >> 2)});
            w.push_back(((b & 1) ? tx : 1.0 - tx) * (((b >> 1) & 1) ? ty : 1.0 - ty) * ((b >> 2) ? tz : 1.0 - tz));
        }
    }
    else
    {
        const int R = p.radius, n = 2 * R + 1;
        const double sigma2 = (p.sigma_cells * c.dx) * (p.sigma_cells * c.dx);
        const int ic = (int)std::floor((e.cx - c.x_min) / c.dx), jc = (int)std::floor((e.cy - c.y_min) / c.dx),
                  kc = (int)std::floor((e.cz - c.z_min) / c.dx);
        for (int t3 = 0; t3 < n * n * n; ++t3)
        {
            const int gi = ic + t3 % n - R, gj = jc + (t3 / n) % n - R, gk = kc + t3 / (n * n) - R;
            const double ddx = c.x_min + (gi + 0.5) * c.dx - e.cx, ddy = c.y_min + (gj + 0.5) * c.dx - e.cy,
                         ddz = c.z_min + (gk + 0.5) * c.dx - e.cz;
            cells.insert(cells.end(), {gi, gj, gk});
            w.push_back(std::exp(-0.5 * (ddx * ddx + ddy * ddy + ddz * ddz) / sigma2));
        }
    }
    bool outside = false, inside = false;
    for (size_t b = 0; b < w.size(); ++b)
    {
        const int gk = cells[3 * b + 2];
        if (gk < 0 || gk >= nzg) continue;
        (gk < k0 || gk >= k1 ? outside : inside) = true;
    }
    if (!outside || !inside) return e;   // the slab's own cells are the whole stencil, or none of it
    double S = 0.0;
    for (size_t b = 0; b < w.size(); ++b)
        if (fluid(cells[3 * b], cells[3 * b + 1], cells[3 * b + 2])) S += w[b];
    if (S < 1e-30) e.mass = 0.0;   // nothing to inject into (06:627)
    else e.wsum = S;
    return e;
}

// Fills the device source schedule with rows for steps [s0, s0 + rows).
int fill_table(lbm_handle* h, long long s0)
{
    const size_t ns = h->srcs.size();
    if (ns == 0) return LBM_OK;
    CK(cudaStreamSynchronize(h->stream), "table refill");   // staging buffer reuse
    for (long long r = 0; r <= kTableRows; ++r)   // rows of steps s0 .. s0 + kTableRows
    {
        const double t = (double)(s0 + r) * h->dt;   // t = s * dt (06:1079)
        for (size_t s = 0; s < ns; ++s) h->h_table[r * ns + s] = entry_for(h, h->srcs[s], t);
    }
    CK(cudaMemcpyAsync(h->d_table, h->h_table, ns * (kTableRows + 1) * sizeof(SourceEntry), cudaMemcpyHostToDevice,
                       h->stream),
       "table upload");
    h->h2d_bytes += (long)(ns * (kTableRows + 1) * sizeof(SourceEntry));
    h->table_base = s0;
    h->table_rows = kTableRows;
    return LBM_OK;
}

int check_ready(lbm_handle* h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    if (!h->inited) return h->fail(LBM_ERR_STATE, "lbm_init has not run");
    return LBM_OK;
}

// Field before the first step: rho is 1 everywhere (06:368) unless
// lbm_set_density gave scheme A an initial pulse, which is then the field at
// FLUID cells (01:197); SOLID cells read 0 as after a step.
void field_rho_initial(const lbm_handle* h, float* out, size_t n)
{
    if (h->rho0.size() != n)
    {
        std::fill(out, out + n, 0.0f);
        return;
    }
    const Layout& L = h->L;
    const size_t nxt = (size_t)L.nx + 2, nyt = (size_t)L.ny + 2;
    size_t c = 0;
    for (int k = 1; k <= L.nz; ++k)
        for (int j = 1; j <= L.ny; ++j)
            for (int i = 1; i <= L.nx; ++i, ++c)
                out[c] = h->mask[(size_t)i + nxt * ((size_t)j + nyt * (size_t)k)] == 1 ? 0.0f : h->rho0[c];
}

// (float)(rho - 1) of the last step into d (device, interior cells).
cudaError_t field_rho_last_step(lbm_handle* h, float* d)
{
    if (!h->scheme_a()) return launch_field_rho(h->storage, h->f[h->cur ^ 1], d, h->L, h->sa, h->scale, h->stream);
    StepArgs sa;
    SchemeAArgs b;
    scheme_a_args(h, h->cur ^ 1, false, h->step - 1, sa, b);
    return launch_field_rho_a((const float*)h->f[h->cur ^ 1], d, h->L, sa, b, h->stream);
}

int reset_halos_if_dirty(lbm_handle* h)
{
    if (!h->halo_dirty) return LBM_OK;
    // All halo cells return to rest (w_q) before the open faces are refilled,
    // as exchange_halos rewrites every halo cell (06:677-682, 06:853-903).
    const Layout& L = h->L;
    const size_t esz = h->storage == LBM_STORE_F16 ? 2 : 4;
    std::vector<double> tmp;   // host round trip is fine: only after lbm_set_f
    const size_t nloc = (size_t)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    double* d = nullptr;
    CK(cudaMalloc(&d, nloc * Q * sizeof(double)), "halo reset");
    cudaError_t e = launch_export_f(h->storage, h->f[h->cur], d, L, h->xf, h->scale, h->stream);
    if (e == cudaSuccess)
    {
        tmp.resize(nloc * Q);
        e = cudaMemcpyAsync(tmp.data(), d, nloc * Q * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    if (e == cudaSuccess)
    {
        const int nxt = L.nx + 2, nyt = L.ny + 2, nzt = L.nz + 2;
        for (int k = 0; k < nzt; ++k)
            for (int j = 0; j < nyt; ++j)
                for (int i = 0; i < nxt; ++i)
                {
                    if (i > 0 && i <= L.nx && j > 0 && j <= L.ny && k > 0 && k <= L.nz) continue;
                    const size_t idx = (size_t)i + (size_t)j * nxt + (size_t)k * nxt * nyt;
                    for (int q = 0; q < Q; ++q) tmp[idx * Q + q] = wd(q);
                }
        e = cudaMemcpyAsync(d, tmp.data(), nloc * Q * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = launch_import_f(h->storage, h->f[h->cur], d, L, h->xf, h->scale, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    cudaFree(d);
    (void)esz;
    if (e != cudaSuccess) return h->cuda_fail(e, "halo reset");
    h->halo_dirty = false;
    return LBM_OK;
}

}  // namespace

// ---------------------------------------------------------------- stepping API

extern "C" int lbm_apply_source(lbm_handle* h, double t)
{
    int st = check_ready(h);
    if (st) return st;
    if (h->srcs.empty()) return LBM_OK;
    if (h->scheme_a()) return LBM_OK;   // scheme A: the field source acts inside lbm_step_collision_bgk
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    SourceArgs a = source_args(h, false);
    for (size_t s = 0; s < h->srcs.size(); ++s) a.direct[s] = entry_for(h, h->srcs[s], t);
    CK(launch_source(h->storage, h->f[h->cur], h->L, h->sa, a, h->stream), "source kernel");
    h->launches++;
    return LBM_OK;
}

extern "C" int lbm_exchange_halos(lbm_handle* h)
{
    int st = check_ready(h);
    if (st) return st;
    if (h->scheme_a()) return LBM_OK;   // scheme A: each step writes the next step's halo values
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    st = reset_halos_if_dirty(h);
    if (st) return st;
    if (h->ga.total > 0)
    {
        CK(launch_ghost(h->storage, h->f[h->cur], h->L, h->ga, h->stream), "ghost kernel");
        h->launches++;
    }
    return LBM_OK;
}

extern "C" int lbm_step_collision_bgk(lbm_handle* h)
{
    int st = check_ready(h);
    if (st) return st;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    CK(timed_step_launch(h, h->cur, false, h->step), "step kernel");
    h->launches++;
    if (h->scheme_a() && h->aa.copy)
    {
        StepArgs sa;
        SchemeAArgs b;
        scheme_a_args(h, h->cur, false, h->step, sa, b);
        CK(launch_copy_a((const float*)h->f[h->cur], (float*)h->f[h->cur ^ 1], h->L, sa, b, h->stream), "halo copy");
        h->launches++;
    }
    h->cur ^= 1;
    h->step++;
    return harvest_timing(h);
}

extern "C" int lbm_record_probes(lbm_handle* h)
{
    int st = check_ready(h);
    if (st) return st;
    if (h->nprobe() == 0) return LBM_OK;
    if (h->step == 0) return h->fail(LBM_ERR_STATE, "no step taken yet");
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    if (h->probe_pending >= kProbeRows)
    {
        st = drain_probes(h);
        if (st) return st;
    }
    // the pre-step buffer of the last collision step is intact until the next one
    if (h->scheme_a())
    {
        StepArgs sa;
        SchemeAArgs b;
        scheme_a_args(h, h->cur ^ 1, false, h->step - 1, sa, b);
        CK(launch_probe_a((const float*)h->f[h->cur ^ 1], h->L, sa, b, probe_args(h, false, h->probe_pending),
                          h->stream),
           "probe kernel");
    }
    else
    {
        CK(launch_probe(h->storage, h->f[h->cur ^ 1], h->L, h->sa, probe_args(h, false, h->probe_pending),
                        h->stream),
           "probe kernel");
    }
    h->launches++;
    h->probe_pending++;
    return LBM_OK;
}

extern "C" int lbm_step(lbm_handle* h, int nsteps)
{
    NvtxRange range("lbm_step");
    int st = check_ready(h);
    if (st) return st;
    if (nsteps < 0) return LBM_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    st = reset_halos_if_dirty(h);
    if (st) return st;
    const int np = h->nprobe();
    const bool use_graph = h->cfg.use_graphs && !h->timing;
    long long left = nsteps;
    while (left > 0)
    {
        if (!h->srcs.empty() && (h->step < h->table_base || h->step >= h->table_base + h->table_rows))
        {
            st = fill_table(h, h->step);
            if (st) return st;
        }
        long long chunk = left;
        if (!h->srcs.empty()) chunk = std::min(chunk, h->table_base + h->table_rows - h->step);
        if (np) chunk = std::min<long long>(chunk, kProbeRows - h->probe_pending);
        if (chunk <= 0)
        {
            st = drain_probes(h);
            if (st) return st;
            continue;
        }
        h->ctl_host->step = h->step;
        h->ctl_host->table_base = h->table_base;
        // the probe row of step s is s - probe_base: rows continue after the
        // ones already buffered
        h->ctl_host->probe_base = h->step - h->probe_pending;
        CK(cudaMemcpyAsync(h->ctl, h->ctl_host, offsetof(Control, nonfinite), cudaMemcpyHostToDevice, h->stream),
           "control");
        h->h2d_bytes += (long)offsetof(Control, nonfinite);
        long long done = 0;
        while (done < chunk)
        {
            if (use_graph && h->cur == 0 && chunk - done >= 2)
            {
                st = build_graph(h);
                if (st) return st;
                CK(cudaGraphLaunch(h->graph, h->stream), "graph launch");
                h->launches += h->graph_kernels;
                done += 2;
            }
            else
            {
                int k = 0;
                CK(enqueue_batched_step(h, h->cur, k), "step launch");
                h->launches += k;
                h->cur ^= 1;
                done += 1;
            }
        }
        if (np)
        {
            // the probe kernels' non-finite flag
            CK(cudaMemcpyAsync(&h->ctl_host->nonfinite, &h->ctl->nonfinite, sizeof(int), cudaMemcpyDeviceToHost,
                               h->stream),
               "probe flag");
            h->d2h_bytes += (long)sizeof(int);
        }
        // the control block upload must not be overwritten before the copy ran
        CK(cudaStreamSynchronize(h->stream), "step sync");
        h->step += chunk;
        if (np) h->probe_pending += chunk;
        left -= chunk;
        if (np && h->ctl_host->nonfinite)
            return h->fail(LBM_ERR_NAN, "non-finite probe value by step " + std::to_string(h->step));
        st = harvest_timing(h);
        if (st) return st;
        if (np && h->probe_pending >= kProbeRows)
        {
            st = drain_probes(h);
            if (st) return st;
        }
    }
    return LBM_OK;
}

extern "C" int lbm_run(lbm_handle* h, double T_total, int frames)
{
    NvtxRange range("lbm_run");
    int st = check_ready(h);
    if (st) return st;
    // 06:1066-1068; steps s = 0..total_steps inclusive (06:1077).
    const int total_steps = (int)std::round(T_total / h->dt);
    const int out_interval = std::max(1, total_steps / std::max(frames, 1));
    if (h->cfg.verbose)
        std::printf("Run: T_total=%g s, Frames=%d, total_steps=%d, out_interval=%d\n", T_total, frames, total_steps,
                    out_interval);
    int left = total_steps + 1;
    while (left > 0)
    {
        const int n = std::min(left, 200);
        st = lbm_step(h, n);
        if (st) return st;
        left -= n;
        if (h->cfg.verbose) std::printf("Step %lld/%d\r", h->step - 1, total_steps);
    }
    if (h->cfg.verbose) std::printf("\nDone.\n");
    return LBM_OK;
}

extern "C" int lbm_synchronize(lbm_handle* h)
{
    int st = check_ready(h);
    if (st) return st;
    CK(cudaStreamSynchronize(h->stream), "synchronize");
    return LBM_OK;
}

// ---------------------------------------------------------------- results

extern "C" int lbm_get_dims(lbm_handle* h, int* n3, int* n3h)
{
    int st = check_ready(h);
    if (st) return st;
    if (n3) { n3[0] = h->NXg; n3[1] = h->NYg; n3[2] = h->NZg; }
    if (n3h) { n3h[0] = h->NXg + 2; n3h[1] = h->NYg + 2; n3h[2] = h->NZg + 2; }
    return LBM_OK;
}

extern "C" double lbm_get_dt(lbm_handle* h)
{
    if (!h) return 0.0;
    return (kCs * h->cfg.dx) / h->cfg.c_phys;
}

extern "C" long lbm_get_step(lbm_handle* h) { return h ? (long)h->step : -1; }

extern "C" int lbm_get_probes(lbm_handle* h, double* out, long capacity, long* nsteps)
{
    int st = check_ready(h);
    if (st) return st;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    st = drain_probes(h);
    const int np = h->nprobe();
    const long rows = np ? (long)(h->series.size() / np) : 0;
    if (nsteps) *nsteps = rows;
    if (!out) return st;
    if ((long)h->series.size() > capacity) return h->fail(LBM_ERR_CAPACITY, "probe buffer too small");
    std::copy(h->series.begin(), h->series.end(), out);
    return st;
}

extern "C" int lbm_get_probe_energy(lbm_handle* h, double* out)
{
    int st = check_ready(h);
    if (st) return st;
    if (!out) return LBM_ERR_INVALID_ARGUMENT;
    const int np = h->nprobe();
    if (np == 0) return LBM_OK;
    CK(cudaMemcpyAsync(out, h->d_energy, (size_t)np * 8, cudaMemcpyDeviceToHost, h->stream), "energy");
    h->d2h_bytes += (long)np * 8;
    CK(cudaStreamSynchronize(h->stream), "energy");
    for (int p = 0; p < np; ++p)
        if (!h->probe_owned[p]) out[p] = NAN;
    return LBM_OK;
}

extern "C" int lbm_get_rho(lbm_handle* h, float* out, long capacity)
{
    int st = check_ready(h);
    if (st) return st;
    const Layout& L = h->L;
    const size_t n = (size_t)L.nx * L.ny * L.nz;
    if (!out || (long)n > capacity) return h->fail(LBM_ERR_CAPACITY, "rho buffer too small");
    if (h->step == 0)
    {
        field_rho_initial(h, out, n);
        return LBM_OK;
    }
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    float* d = nullptr;
    CK(cudaMalloc(&d, n * sizeof(float)), "rho buffer");
    cudaError_t e = field_rho_last_step(h, d);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    h->d2h_bytes += (long)(n * sizeof(float));
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return h->cuda_fail(e, "get_rho");
    h->launches++;
    return LBM_OK;
}

// Same output as lbm_get_rho without any device allocation: the field goes
// through the library's statically reserved array (see nlos_lbm.h).
extern "C" int lbm_get_rho_noalloc(lbm_handle* h, float* out, long capacity)
{
    int st = check_ready(h);
    if (st) return st;
    const Layout& L = h->L;
    const long long n = (long long)L.nx * L.ny * L.nz;
    if (n > LBM_NOALLOC_MAX_CELLS)
        return h->fail(LBM_ERR_UNSUPPORTED, "lbm_get_rho_noalloc: the grid has " + std::to_string(n) +
                                                " cells; the static field array holds at most " +
                                                std::to_string((long long)LBM_NOALLOC_MAX_CELLS));
    if (!out || (long long)capacity < n) return h->fail(LBM_ERR_CAPACITY, "rho buffer too small");
    if (h->step == 0)
    {
        field_rho_initial(h, out, (size_t)n);
        return LBM_OK;
    }
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    float* d = nullptr;
    CK(field_scratch_address(h->device, &d), "static field array address");
    // every cell of the first n entries is written by the kernel: nothing to clear
    CK(field_rho_last_step(h, d), "field kernel");
    CK(cudaMemcpyAsync(out, d, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "field download");
    CK(cudaStreamSynchronize(h->stream), "field download");
    h->launches++;
    h->d2h_bytes += (long)(n * (long long)sizeof(float));
    return LBM_OK;
}

extern "C" int lbm_get_f(lbm_handle* h, double* out, long capacity)
{
    int st = check_ready(h);
    if (st) return st;
    const Layout& L = h->L;
    const size_t n = (size_t)(L.nx + 2) * (L.ny + 2) * (L.nz + 2) * Q;
    if (h->scheme_a()) return h->fail(LBM_ERR_UNSUPPORTED, "scheme A stores post-collision populations; use lbm_get_rho");
    if (!out || (long)n > capacity) return h->fail(LBM_ERR_CAPACITY, "f buffer too small");
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    double* d = nullptr;
    CK(cudaMalloc(&d, n * sizeof(double)), "f export buffer");
    cudaError_t e = launch_export_f(h->storage, h->f[h->cur], d, L, h->xf, h->scale, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    h->d2h_bytes += (long)(n * sizeof(double));
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return h->cuda_fail(e, "get_f");
    h->launches++;
    return LBM_OK;
}

extern "C" int lbm_set_f(lbm_handle* h, const double* in, long count)
{
    int st = check_ready(h);
    if (st) return st;
    const Layout& L = h->L;
    const size_t n = (size_t)(L.nx + 2) * (L.ny + 2) * (L.nz + 2) * Q;
    if (h->scheme_a()) return h->fail(LBM_ERR_UNSUPPORTED, "scheme A state cannot be set from f");
    if (!in || count != (long)n) return h->fail(LBM_ERR_INVALID_ARGUMENT, "f size mismatch");
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    double* d = nullptr;
    CK(cudaMalloc(&d, n * sizeof(double)), "f import buffer");
    cudaError_t e = cudaMemcpyAsync(d, in, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    h->h2d_bytes += (long)(n * sizeof(double));
    if (e == cudaSuccess) e = launch_import_f(h->storage, h->f[h->cur], d, L, h->xf, h->scale, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return h->cuda_fail(e, "set_f");
    h->launches++;
    h->halo_dirty = true;
    return LBM_OK;
}

extern "C" int lbm_set_density(lbm_handle* h, const double* rho_minus_1, long count)
{
    int st = check_ready(h);
    if (st) return st;
    const Layout& L = h->L;
    const size_t n = (size_t)L.nx * L.ny * L.nz;
    if (!h->scheme_a()) return h->fail(LBM_ERR_UNSUPPORTED, "lbm_set_density sets the scheme-A state");
    if (h->step != 0) return h->fail(LBM_ERR_STATE, "lbm_set_density before the first step");
    if (!rho_minus_1 || count != (long)n) return h->fail(LBM_ERR_INVALID_ARGUMENT, "density size mismatch");
    std::vector<float> rp(n);
    for (size_t i = 0; i < n; ++i) rp[i] = (float)rho_minus_1[i];
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    float* d_rp = nullptr;
    uint8_t* d_mask = nullptr;
    cudaError_t e = cudaMalloc(&d_rp, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_mask, h->mask.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rp, rp.data(), n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_mask, h->mask.data(), h->mask.size(), cudaMemcpyHostToDevice, h->stream);
    h->h2d_bytes += (long)(n * sizeof(float) + h->mask.size());
    if (e == cudaSuccess)
        e = launch_set_density_a((float*)h->f[h->cur], h->xgh_par[h->cur], d_rp, d_mask, L, h->aa, h->stream);
    if (e == cudaSuccess && h->aa.zper) e = launch_zper_a((float*)h->f[h->cur], L, h->sa, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_rp);
    cudaFree(d_mask);
    if (e != cudaSuccess) return h->cuda_fail(e, "set_density");
    h->rho0 = std::move(rp);
    h->launches += h->aa.zper ? 2 : 1;
    return LBM_OK;
}

extern "C" int lbm_get_mask(lbm_handle* h, uint8_t* out, long capacity)
{
    int st = check_ready(h);
    if (st) return st;
    if (!out || (long)h->mask.size() > capacity) return h->fail(LBM_ERR_CAPACITY, "mask buffer too small");
    std::copy(h->mask.begin(), h->mask.end(), out);
    return LBM_OK;
}

// ---------------------------------------------------------------- measurement

extern "C" int lbm_set_kernel_timing(lbm_handle* h, int enable)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    h->timing = enable != 0;
    h->kernel_ms = 0.0;
    h->kernel_launches = 0;
    h->ev_used = 0;
    return LBM_OK;
}

extern "C" int lbm_get_kernel_time(lbm_handle* h, double* total_ms, long* launches)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    int st = harvest_timing(h);
    if (total_ms) *total_ms = h->kernel_ms;
    if (launches) *launches = h->kernel_launches;
    return st;
}

extern "C" long lbm_get_launch_count(lbm_handle* h) { return h ? h->launches : -1; }

extern "C" void* lbm_get_stream(lbm_handle* h) { return h ? (void*)h->stream : nullptr; }

extern "C" int lbm_get_transfer_bytes(lbm_handle* h, long* h2d, long* d2h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    if (h2d) *h2d = h->h2d_bytes;
    if (d2h) *d2h = h->d2h_bytes;
    return LBM_OK;
}

extern "C" int lbm_check_status(lbm_handle* h, long long* site, long long* index)
{
    if (!h || !site || !index) return LBM_ERR_INVALID_ARGUMENT;
#ifndef LBM_CHECK
    return h->fail(LBM_ERR_UNSUPPORTED, "bounds checks are compiled only into liblbm_b200_check.so");
#else
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    if (h->stream) CK(cudaStreamSynchronize(h->stream), "check status");
    *site = 0;
    *index = 0;
    check::Status st[3];
    CK(check_read_kernels(&st[0]), "check status");
    CK(check_read_adjoint(&st[1]), "check status");
    CK(check_read_scheme_a(&st[2]), "check status");
    for (const check::Status& c : st)
        if (c.site != 0 && *site == 0)
        {
            *site = c.site;
            *index = c.index;
        }
    return LBM_OK;
#endif
}

extern "C" int lbm_check_selftest(lbm_handle* h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
#ifndef LBM_CHECK
    return h->fail(LBM_ERR_UNSUPPORTED, "bounds checks are compiled only into liblbm_b200_check.so");
#else
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    CK(launch_check_selftest(h->stream), "check self-test");
    CK(cudaStreamSynchronize(h->stream), "check self-test");
    return LBM_OK;
#endif
}

extern "C" int lbm_bytes_per_cell(lbm_handle* h)
{
    if (!h) return 0;
    return 2 * Q * (h->storage == LBM_STORE_F16 ? 2 : 4);
}

// ---------------------------------------------------------------- synthetic geometry

extern "C" int lbm_city_generate(const lbm_city_params* p, float* tris, int capacity, int* ntris, double* coverage)
{
    if (!p || !ntris) return LBM_ERR_INVALID_ARGUMENT;
    if (p->nx <= 0 || p->ny <= 0 || p->fp_min <= 0 || p->fp_max < p->fp_min || p->h_min <= 0 ||
        p->h_max < p->h_min || p->street < 0 || p->margin < 0 || !(p->dx > 0))
        return LBM_ERR_INVALID_ARGUMENT;
    std::vector<float> t;
    const double cov = city_generate(*p, t);
    const int n = (int)(t.size() / 9);
    *ntris = n;
    if (coverage) *coverage = cov;
    if (!tris || capacity < n) return LBM_ERR_CAPACITY;
    std::copy(t.begin(), t.end(), tris);
    return LBM_OK;
}

extern "C" int lbm_stl_write(const char* path, const float* tris, int ntris)
{
    if (!path || ntris < 0 || (ntris > 0 && !tris)) return LBM_ERR_INVALID_ARGUMENT;
    return stl_write(path, tris, ntris) ? LBM_OK : LBM_ERR_IO;
}

extern "C" int lbm_voxelize(const lbm_config* cfg, const float* tris, int ntris, double scale, double sx, double sy,
                            double sz, uint8_t* mask, long capacity, int* n3_halo)
{
    if (!cfg || ntris < 0 || (ntris > 0 && !tris)) return LBM_ERR_INVALID_ARGUMENT;
    std::string why;
    if (validate(*cfg, why) != LBM_OK) return LBM_ERR_BAD_CONFIG;
    int nx, ny, nz;
    grid_size(*cfg, nx, ny, nz);
    if (nx < 1 || ny < 1 || nz < 1) return LBM_ERR_BAD_CONFIG;
    if (n3_halo)
    {
        n3_halo[0] = nx + 2; n3_halo[1] = ny + 2; n3_halo[2] = nz + 2;
    }
    const long n = (long)(nx + 2) * (ny + 2) * (nz + 2);
    if (!mask || capacity < n) return LBM_ERR_CAPACITY;
    HeightField geo;
    geo.set_triangles(tris, ntris, scale, sx, sy, sz);
    build_mask(*cfg, geo, nx, ny, nz, mask);
    return LBM_OK;
}

// ---------------------------------------------------------------- adjoint

namespace {

// Sub-allocations of the adjoint workspace, 256-byte aligned.  With a null
// base it only counts the bytes.
struct Carve
{
    char* base = nullptr;
    size_t used = 0;
    template <typename T>
    T* get(size_t n)
    {
        T* p = base ? (T*)(base + used) : nullptr;
        used += (std::max<size_t>(n, 1) * sizeof(T) + 255) / 256 * 256;
        return p;
    }
};

// n stored forward states, each a population buffer plus one x-face array
// (the x-face exports for a checkpoint of G, the x-face ghosts for a stored Ht).
struct StateSlots
{
    float* base = nullptr;
    size_t pop = 0, face = 0;   // floats, rounded up to 64
    float* pop_of(long long s) const { return base + (size_t)s * (pop + face); }
    float* face_of(long long s) const { return pop_of(s) + pop; }
};

// All lattice cells are back at rest and the step counter at 0.
int rest_state(lbm_handle* h)
{
    const size_t pop_bytes = (size_t)h->L.total * (h->storage == LBM_STORE_F16 ? 2 : 4);
    const size_t n_xexp = (size_t)2 * Q * h->L.ny * h->L.nz, n_xgh = (size_t)2 * Q * (h->L.ny + 2) * (h->L.nz + 2);
    for (int b = 0; b < 2; ++b) CK(cudaMemsetAsync(h->f[b], 0, pop_bytes, h->stream), "rest state");
    CK(cudaMemsetAsync(h->xf.xexp, 0, n_xexp * sizeof(float), h->stream), "rest state");
    CK(cudaMemsetAsync(h->xf.xgh, 0, n_xgh * sizeof(float), h->stream), "rest state");
    CK(cudaMemsetAsync(h->d_energy, 0, (size_t)std::max(h->nprobe(), 1) * sizeof(double), h->stream), "rest state");
    CK(cudaStreamSynchronize(h->stream), "rest state");
    h->step = 0;
    h->cur = 0;
    h->series.clear();
    h->probe_pending = 0;
    h->halo_dirty = false;
    return LBM_OK;
}

// Injection cells of the single source at one step with their normalised
// weights and the weights' derivatives with respect to the source position
// (metres).  Same cell set, fluid test and normalisation as k_source.
void source_cells(const lbm_handle* h, const lbm_source& p, const SourceEntry& e, int ncell, AdjSourceCell* out)
{
    const lbm_config& c = h->cfg;
    const Layout& L = h->L;
    const int nxt = L.nx + 2, nyt = L.ny + 2;
    std::vector<double> ww((size_t)ncell, 0.0), dw((size_t)ncell * 3, 0.0);
    std::vector<int> ijk((size_t)ncell * 3, 0);
    std::vector<char> fluid((size_t)ncell, 0);
    for (int b = 0; b < ncell; ++b) out[b] = AdjSourceCell{-1, 0, 0, 0, 0.0, {0.0, 0.0, 0.0}};
    const auto is_fluid = [&](int gi, int gj, int gk) {
        if (gi < 0 || gi >= L.nx || gj < 0 || gj >= L.ny || gk < 0 || gk >= L.nz) return false;
        return h->mask[(size_t)(gi + 1) + (size_t)(gj + 1) * nxt + (size_t)(gk + 1) * nxt * nyt] == 0;
    };
    if (p.injection == LBM_INJECT_TRILINEAR)
    {
        const double fx = (e.cx - c.x_min) / c.dx - 0.5;
        const double fy = (e.cy - c.y_min) / c.dx - 0.5;
        const double fz = (e.cz - c.z_min) / c.dx - 0.5;
        const int i0 = (int)std::floor(fx), j0 = (int)std::floor(fy), k0 = (int)std::floor(fz);
        const double tx = fx - i0, ty = fy - j0, tz = fz - k0;
        for (int b = 0; b < 8; ++b)
        {
            const int bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
            const double wx = bx ? tx : 1.0 - tx, wy = by ? ty : 1.0 - ty, wz = bz ? tz : 1.0 - tz;
            const double sx = (bx ? 1.0 : -1.0) / c.dx, sy = (by ? 1.0 : -1.0) / c.dx, sz = (bz ? 1.0 : -1.0) / c.dx;
            ijk[3 * b] = i0 + bx;
            ijk[3 * b + 1] = j0 + by;
            ijk[3 * b + 2] = k0 + bz;
            ww[b] = wx * wy * wz;
            dw[3 * b] = sx * wy * wz;
            dw[3 * b + 1] = wx * sy * wz;
            dw[3 * b + 2] = wx * wy * sz;
            fluid[b] = is_fluid(ijk[3 * b], ijk[3 * b + 1], ijk[3 * b + 2]);
        }
    }
    else
    {
        const int R = p.radius, n = 2 * R + 1;
        const double sigma2 = (p.sigma_cells * c.dx) * (p.sigma_cells * c.dx);
        const int ic = (int)std::floor((e.cx - c.x_min) / c.dx);
        const int jc = (int)std::floor((e.cy - c.y_min) / c.dx);
        const int kc = (int)std::floor((e.cz - c.z_min) / c.dx);
        if (ic < -R || ic >= L.nx + R || jc < -R || jc >= L.ny + R || kc < -R || kc >= L.nz + R) return;
        for (int b = 0; b < ncell; ++b)
        {
            const int gi = ic + b % n - R, gj = jc + (b / n) % n - R, gk = kc + b / (n * n) - R;
            const double x = c.x_min + (gi + 0.5) * c.dx, y = c.y_min + (gj + 0.5) * c.dx,
                         z = c.z_min + (gk + 0.5) * c.dx;
            const double ddx = x - e.cx, ddy = y - e.cy, ddz = z - e.cz;
            const double w = std::exp(-0.5 * (ddx * ddx + ddy * ddy + ddz * ddz) / sigma2);
            ijk[3 * b] = gi;
            ijk[3 * b + 1] = gj;
            ijk[3 * b + 2] = gk;
            ww[b] = w;
            dw[3 * b] = w * ddx / sigma2;   // d/dcx exp(-(x-cx)^2 / 2s^2)
            dw[3 * b + 1] = w * ddy / sigma2;
            dw[3 * b + 2] = w * ddz / sigma2;
            fluid[b] = is_fluid(gi, gj, gk);
        }
    }
    double S = 0.0, dS[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < ncell; ++b)
        if (fluid[b])
        {
            S += ww[b];
            for (int a = 0; a < 3; ++a) dS[a] += dw[3 * b + a];
        }
    if (S < 1e-30) return;
    for (int b = 0; b < ncell; ++b)
    {
        if (!fluid[b]) continue;
        AdjSourceCell& o = out[b];
        o.i = ijk[3 * b] + 1;
        o.j = ijk[3 * b + 1] + 1;
        o.k = ijk[3 * b + 2] + 1;
        o.what = ww[b] / S;
        for (int a = 0; a < 3; ++a) o.dwhat[a] = (dw[3 * b + a] * S - ww[b] * dS[a]) / (S * S);
    }
}

// Checkpoint schedule of one adjoint evaluation: outer interval K1, inner
// interval K2 and the device bytes it allocates.  ckpt_inner <= 0 picks the
// largest K2 <= K1 whose buffers fit in 90 % of the free device memory and
// then, within the same budget, the longest tail of whole outer segments
// [Tt, T) whose forward data the first pass stores (those segments are
// reversed without a recompute).
struct AdjPlan
{
    int K1 = 0, K2 = 0, M = 0, NI = 0, ncell = 0;
    int Tt = 0;                                  // tail start (T: no tail), a multiple of K1
    int C = 0;                                   // store slots (steps of forward data)
    size_t pop = 0, ck_slot = 0, st_slot = 0;   // floats; st_slot: one step's stored moments
    size_t mom_n = 0;                            // 4-byte words of pair moments per stored step
    long long gadj_n = 0;
    size_t bytes = 0;
    long long fwd_steps = 0;                     // forward steps run, recomputation included
};

size_t round64(size_t n) { return (n + 63) / 64 * 64; }

AdjPlan adjoint_plan(const lbm_handle* h, int T, int ckpt_outer, int ckpt_inner)
{
    AdjPlan p;
    const Layout& L = h->L;
    const lbm_source& s = h->srcs[0].s;
    p.ncell = s.injection == LBM_INJECT_TRILINEAR ? 8 : (2 * s.radius + 1) * (2 * s.radius + 1) * (2 * s.radius + 1);
    p.pop = round64((size_t)L.total);
    p.ck_slot = p.pop + round64((size_t)2 * Q * L.ny * L.nz);
    // stored per step: moments of F^s for every cell (two FP16 pairs), moments of H^s at every ghost's interior cell (FP32)
    p.mom_n = round64((size_t)((L.nx + 1) / 2) * L.ny * L.nz * (sizeof(PairMoments) / 4));
    p.st_slot = p.mom_n + 4 * round64((size_t)std::max(h->ga.total, 1LL));   // 12-bit cell moments, FP32 faces
    for (int f = 0; f < h->ga.nfaces; ++f) p.gadj_n += (long long)Q * h->ga.face[f].nu * h->ga.face[f].nv;
    p.K1 = std::min(ckpt_outer > 0 ? ckpt_outer : 200, T);
    p.M = (T + p.K1 - 1) / p.K1;
    const int np = h->nprobe();
    // Mr: outer segments reversed with a recompute (those before the tail); only they
    // need a full-state checkpoint and, when there is one, the inner checkpoints
    const auto bytes = [&](int K2, int C, int Mr) {
        const size_t ni = Mr > 0 ? (size_t)((p.K1 + K2 - 1) / K2) : 0;
        Carve c;
        c.get<float>((size_t)Mr * p.ck_slot);
        c.get<float>(ni * p.ck_slot);
        c.get<float>((size_t)std::max(C, K2 + 1) * p.st_slot);
        c.get<float>(p.pop);
        c.get<float>(p.pop);
        c.get<float>((size_t)p.gadj_n);
        c.get<double>((size_t)T * np);
        c.get<double>((size_t)T * np);
        c.get<AdjSourceCell>((size_t)T * p.ncell);
        c.get<double>((size_t)T * 4);
        return c.used;
    };
    p.Tt = T;
    if (ckpt_inner > 0)
    {
        p.K2 = std::min(ckpt_inner, p.K1);
    }
    else
    {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
        double budget = 0.9 * (double)(fr + h->adj_ws_bytes);   // the workspace is reused
        // NLOS_LBM_ADJ_BUDGET: a smaller cap in bytes (e.g. for a GPU shared with other work)
        if (const char* v = std::getenv("NLOS_LBM_ADJ_BUDGET")) budget = std::min(budget, std::atof(v));
        p.K2 = 1;
        for (int K2 = p.K1; K2 >= 1; --K2)
            if ((double)bytes(K2, K2 + 1, p.M) <= budget)
            {
                p.K2 = K2;
                break;
            }
        // the tail: steps max(Tt - 1, 0) .. T - 1 keep their forward data
        for (int m = 0; m < p.M; ++m)
        {
            const int Tt = m * p.K1, need = T - std::max(Tt - 1, 0);
            if ((double)bytes(p.K2, need, m) <= budget)
            {
                p.Tt = Tt;
                break;
            }
        }
    }
    p.C = std::max(p.K2 + 1, T - std::max(p.Tt - 1, 0));
    if (p.Tt == T) p.C = p.K2 + 1;
    p.NI = (p.K1 + p.K2 - 1) / p.K2;
    p.bytes = bytes(p.K2, p.C, (p.Tt + p.K1 - 1) / p.K1);
    // forward steps (fused pull-collide launches): the first pass, the outer
    // recompute to the inner checkpoints and the recompute of every inner
    // segment before the tail (its last state needs only the source and ghost fill)
    p.fwd_steps = T;
    for (int m = 0; m < p.M && m * p.K1 < p.Tt; ++m)
    {
        const long long O = (long long)m * p.K1, E = std::min<long long>(O + p.K1, T);
        const long long N = (E - O + p.K2 - 1) / p.K2;
        p.fwd_steps += std::max(O + (N - 1) * p.K2 - 1, 0LL) - std::max(O - 1, 0LL);
        for (long long n = 0; n < N; ++n)
        {
            const long long a0 = O + n * p.K2, a1 = std::min(a0 + p.K2, E);
            p.fwd_steps += a1 - 1 - std::max(a0 - 1, 0LL);
        }
    }
    return p;
}

}  // namespace

extern "C" int lbm_adjoint_release(lbm_handle* h)
{
    if (!h) return LBM_ERR_INVALID_ARGUMENT;
    if (h->adj_ws)
    {
        CK(cudaSetDevice(h->device), "cudaSetDevice");
        CK(cudaStreamSynchronize(h->stream), "adjoint release");
        cudaFree(h->adj_ws);
    }
    h->adj_ws = nullptr;
    h->adj_ws_bytes = 0;
    return LBM_OK;
}

extern "C" int lbm_adjoint_plan(lbm_handle* h, int nsteps, int ckpt_outer, int ckpt_inner, int* outer, int* inner,
                                long long* device_bytes, long long* forward_steps)
{
    int st = check_ready(h);
    if (st) return st;
    if (h->srcs.size() != 1) return h->fail(LBM_ERR_UNSUPPORTED, "the adjoint needs exactly one source");
    if (nsteps < 1) return h->fail(LBM_ERR_INVALID_ARGUMENT, "nsteps < 1");
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    const AdjPlan p = adjoint_plan(h, nsteps, ckpt_outer, ckpt_inner);
    if (outer) *outer = p.K1;
    if (inner) *inner = p.K2;
    if (device_bytes) *device_bytes = (long long)p.bytes;
    if (forward_steps) *forward_steps = p.fwd_steps;
    return LBM_OK;
}

extern "C" int lbm_adjoint_grad(lbm_handle* h, int nsteps, const double* observed, int ckpt_outer, int ckpt_inner,
                                double* loss, double* grad_pos, double* grad_signal, double* predicted)
{
    NvtxRange range("lbm_adjoint_grad");
    int st = check_ready(h);
    if (st) return st;
    if (h->storage != LBM_STORE_F32) return h->fail(LBM_ERR_UNSUPPORTED, "the adjoint runs on FP32 storage");
    if (h->scheme_a()) return h->fail(LBM_ERR_UNSUPPORTED, "the adjoint differentiates scheme B");
    if (h->slab) return h->fail(LBM_ERR_UNSUPPORTED, "the adjoint runs on a whole grid, not a z-slab");
    if (h->srcs.size() != 1) return h->fail(LBM_ERR_UNSUPPORTED, "the adjoint needs exactly one source");
    const int np = h->nprobe();
    if (np < 1) return h->fail(LBM_ERR_STATE, "the adjoint needs probes");
    if (nsteps < 1 || !observed || !loss) return h->fail(LBM_ERR_INVALID_ARGUMENT, "nsteps, observed or loss");
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    st = rest_state(h);
    if (st) return st;

    const int T = nsteps;
    const AdjPlan plan = adjoint_plan(h, T, ckpt_outer, ckpt_inner);
    const int K1 = plan.K1, K2 = plan.K2, NI = plan.NI, ncell = plan.ncell;
    const int Tt = plan.Tt;                        // steps Tt .. T-1 are reversed from the first pass's data
    const int Mr = (Tt + K1 - 1) / K1;             // outer segments reversed with a recompute
    const Layout& L = h->L;
    const size_t n_xexp = (size_t)2 * Q * L.ny * L.nz;
    const size_t pop = plan.pop;
    const SourceState& src = h->srcs[0];

    // Source schedule and injection cells of every step (host, FP64).
    std::vector<SourceEntry> entries((size_t)T);
    std::vector<AdjSourceCell> cells((size_t)T * ncell);
    for (int s = 0; s < T; ++s)
    {
        entries[s] = source_entry(src, (double)s * h->dt, h->dt);
        source_cells(h, src.s, entries[s], ncell, &cells[(size_t)s * ncell]);
    }

    // Open faces of the ghost adjoint.
    long long gadj_off[6] = {-1, -1, -1, -1, -1, -1};
    long long gadj_n = 0;
    for (int f = 0; f < h->ga.nfaces; ++f)
    {
        const GhostFace& F = h->ga.face[f];
        gadj_off[F.axis * 2 + F.side] = gadj_n;
        gadj_n += (long long)Q * F.nu * F.nv;
    }

    // workspace: carved from one allocation kept in the handle between calls
    StateSlots outer, inner;
    float* store;
    float* lam[2];
    float* gadj;
    double *d_pred, *d_resid, *d_out;
    AdjSourceCell* d_cells;
    const auto carve = [&](Carve& c) {
        outer = StateSlots{c.get<float>((size_t)Mr * plan.ck_slot), pop, plan.ck_slot - pop};
        inner = StateSlots{c.get<float>((size_t)(Mr > 0 ? NI : 0) * plan.ck_slot), pop, plan.ck_slot - pop};
        store = c.get<float>((size_t)plan.C * plan.st_slot);
        lam[0] = c.get<float>(pop);
        lam[1] = c.get<float>(pop);
        gadj = c.get<float>((size_t)gadj_n);
        d_pred = c.get<double>((size_t)T * np);
        d_resid = c.get<double>((size_t)T * np);
        d_cells = c.get<AdjSourceCell>(cells.size());
        d_out = c.get<double>((size_t)T * 4);
    };
    {
        Carve count;
        carve(count);
        if (count.used > h->adj_ws_bytes)
        {
            if (h->adj_ws) cudaFree(h->adj_ws);
            h->adj_ws = nullptr;
            h->adj_ws_bytes = 0;
            CK(cudaMalloc(&h->adj_ws, count.used), "adjoint workspace");
            h->adj_ws_bytes = count.used;
        }
        Carve c{(char*)h->adj_ws, 0};
        carve(c);
    }
    const auto mom_of = [&](long long slot) { return (PairMoments*)(store + (size_t)slot * plan.st_slot); };
    const auto face_mom_of = [&](long long slot) {
        return (float4*)(store + (size_t)slot * plan.st_slot + plan.mom_n);
    };
    CK(cudaMemcpyAsync(d_cells, cells.data(), cells.size() * sizeof(AdjSourceCell), cudaMemcpyHostToDevice, h->stream),
       "adjoint upload");
    CK(cudaMemsetAsync(d_out, 0, (size_t)T * 4 * sizeof(double), h->stream), "adjoint memset");
    const size_t pop_bytes = (size_t)L.total * sizeof(float);
    SourceArgs sargs = source_args(h, false);
    // L2 prefetch distance of the adjoint step in rows (NLOS_LBM_ADJ_PREFETCH_ROWS, 0 = off)
    int adj_prefetch = kDefaultAdjointPrefetchRows;
    if (const char* v = std::getenv("NLOS_LBM_ADJ_PREFETCH_ROWS")) adj_prefetch = std::max(0, std::atoi(v));
    long kernels = 0;
    const auto save_g = [&](const StateSlots& sl, long long idx) {
        cudaError_t r = cudaMemcpyAsync(sl.pop_of(idx), h->f[h->cur], pop_bytes, cudaMemcpyDeviceToDevice, h->stream);
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(sl.face_of(idx), h->xf.xexp, n_xexp * sizeof(float), cudaMemcpyDeviceToDevice,
                                h->stream);
        return r;
    };
    const auto restore_g = [&](const StateSlots& sl, long long idx) {
        h->cur = 0;
        cudaError_t r = cudaMemcpyAsync(h->f[0], sl.pop_of(idx), pop_bytes, cudaMemcpyDeviceToDevice, h->stream);
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(h->xf.xexp, sl.face_of(idx), n_xexp * sizeof(float), cudaMemcpyDeviceToDevice,
                                h->stream);
        return r;
    };
    // The ghost fill reads only the first interior layer of each open face (the
    // x faces through their export arrays, which the source also updates);
    // when step s's injection cells stay off that layer, source and ghost fill
    // touch disjoint cells and the source runs on the side stream beside it.
    std::vector<char> source_apart((size_t)T, 0);
    for (int s = 0; s < T; ++s)
    {
        bool apart = true;
        for (int b = 0; b < ncell && apart; ++b)
        {
            const AdjSourceCell& cc = cells[(size_t)s * ncell + b];
            if (cc.i < 0) continue;
            for (int f = 0; f < h->ga.nfaces; ++f)
            {
                const GhostFace& F = h->ga.face[f];
                const int v = F.axis == 0 ? cc.i : F.axis == 1 ? cc.j : cc.k;
                const int n = F.axis == 0 ? L.nx : F.axis == 1 ? L.ny : L.nz;
                if (v == (F.side ? n : 1)) apart = false;
            }
        }
        source_apart[(size_t)s] = apart;
    }
    // source + ghost fill of step s on the current buffer (G^s -> Ht^s)
    const auto source_then_ghost = [&](int s, const GhostArgs& g) {
        sargs.direct[0] = entries[s];
        cudaError_t r = cudaSuccess;
        const bool beside = h->ga.total > 0 && source_apart[(size_t)s];
        if (beside)
        {
            r = cudaEventRecord(h->ev_fork, h->stream);
            if (r == cudaSuccess) r = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
            if (r == cudaSuccess) r = launch_source(h->storage, h->f[h->cur], L, h->sa, sargs, h->side);
            if (r == cudaSuccess) r = cudaEventRecord(h->ev_join, h->side);
        }
        else
        {
            r = launch_source(h->storage, h->f[h->cur], L, h->sa, sargs, h->stream);
        }
        kernels++;
        if (r == cudaSuccess && h->ga.total > 0)
        {
            r = launch_ghost(h->storage, h->f[h->cur], L, g, h->stream);
            kernels++;
        }
        if (r == cudaSuccess && beside) r = cudaStreamWaitEvent(h->stream, h->ev_join, 0);
        return r;
    };
    const auto source_ghost = [&](int s) { return source_then_ghost(s, h->ga); };
    // pull + collide of step s (Ht^s -> G^{s+1}), optionally with its probe record
    // The probe record of step s reads the step's input buffer, which the step
    // only reads: it runs on the side stream beside the step, joined before
    // anything can overwrite that buffer (the next step writes into it).
    const auto probe_beside = [&](int s) {
        ProbeArgs pa = probe_args(h, false, s);
        pa.out = d_pred;
        cudaError_t r = cudaEventRecord(h->ev_fork, h->stream);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
        if (r == cudaSuccess) r = launch_probe(h->storage, h->f[h->cur], L, h->sa, pa, h->side);
        if (r == cudaSuccess) r = cudaEventRecord(h->ev_join, h->side);
        kernels++;
        return r;
    };
    const auto collide = [&](int s, bool probe) {
        cudaError_t r = probe ? probe_beside(s) : cudaSuccess;
        if (r == cudaSuccess)
            r = launch_step(h->storage, h->f[h->cur], h->f[h->cur ^ 1], L, h->sa, h->scale, h->stream);
        kernels++;
        if (r == cudaSuccess && probe) r = cudaStreamWaitEvent(h->stream, h->ev_join, 0);
        h->cur ^= 1;
        return r;
    };
    // Recompute of step s for the reverse pass: source and ghost fill
    // recording the moments of H^s at the ghosts' interior cells, then the
    // fused step recording the moments of F^s, both into store slot `slot`.
    const auto stored_source_ghost = [&](int s, long long slot) {
        GhostArgs g = h->ga;
        g.face_mom = face_mom_of(slot);
        return source_then_ghost(s, g);
    };
    // probe_step >= 0: also the probe record of that step (first pass)
    const auto stored_collide = [&](long long slot, int probe_step = -1) {
        kernels++;
        cudaError_t r = probe_step >= 0 ? probe_beside(probe_step) : cudaSuccess;
        if (r == cudaSuccess)
            r = launch_step_moments((const float*)h->f[h->cur], (float*)h->f[h->cur ^ 1], L, h->sa, mom_of(slot),
                                    h->stream);
        if (r == cudaSuccess && probe_step >= 0) r = cudaStreamWaitEvent(h->stream, h->ev_join, 0);
        h->cur ^= 1;
        return r;
    };
    const auto ckpt_pos = [&](long long boundary) { return std::max(boundary - 1, 0LL); };
    const long long cnT = ckpt_pos(Tt);   // first step whose forward data the first pass stores

    // ---- forward pass: probe predictions, outer checkpoints G^{max(mK1-1,0)}
    // of the segments before the tail, and the tail's forward data
    {
        NvtxRange phase("adjoint forward pass");
        int m = 0;
        for (int s = 0; s < T; ++s)
        {
            while (m < Mr && ckpt_pos((long long)m * K1) == s)
            {
                CK(save_g(outer, m), "checkpoint");
                ++m;
            }
            if (Tt < T && s >= cnT)
            {
                CK(stored_source_ghost(s, s - cnT), "adjoint forward");
                CK(stored_collide(s - cnT, s), "adjoint forward");
            }
            else
            {
                CK(source_ghost(s), "adjoint forward");
                CK(collide(s, true), "adjoint forward");
            }
        }
    }

    // ---- misfit (FP64 on the host) and residuals
    std::vector<double> pred((size_t)T * np), resid((size_t)T * np, 0.0);
    CK(cudaMemcpyAsync(pred.data(), d_pred, pred.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
       "prediction download");
    CK(cudaStreamSynchronize(h->stream), "prediction download");
    double Lsum = 0.0;
    for (int s = 0; s < T; ++s)
        for (int p = 0; p < np; ++p)
        {
            const size_t n = (size_t)s * np + p;
            if (!h->probe_owned[p] || !std::isfinite(observed[n])) continue;
            if (!std::isfinite(pred[n])) return h->fail(LBM_ERR_NAN, "non-finite forward probe value");
            const double r = pred[n] - observed[n];
            Lsum += 0.5 * r * r;
            if (!h->probe_solid[p]) resid[n] = r;   // a SOLID probe reads 0 whatever the state
        }
    CK(cudaMemcpyAsync(d_resid, resid.data(), resid.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream),
       "residual upload");

    // ---- reverse pass
    NvtxRange reverse_phase("adjoint reverse pass");
    for (int b = 0; b < 2; ++b) CK(cudaMemsetAsync(lam[b], 0, pop * sizeof(float), h->stream), "adjoint memset");
    int la = 0;
    AdjProbeArgs pa{np, h->d_probe_ijk, nullptr, L};
    pa.resid = d_resid + (size_t)(T - 1) * np;
    CK(launch_adj_probe(lam[la], pa, h->stream), "adjoint probe");
    kernels++;
    // adjoint steps a1-1 .. a0 with the forward data of step s in store slot s - cn
    const auto reverse_segment = [&](int a0, int a1, int cn) -> int {
        for (int s = a1 - 1; s >= a0; --s)
        {
            if (h->ga.total > 0)
            {
                AdjGhostArgs ga{L, h->ga, h->links, lam[la], face_mom_of(s - cn), gadj, {}};
                std::copy(gadj_off, gadj_off + 6, ga.gadj_off);
                CK(launch_adj_ghost(ga, h->stream), "adjoint ghost");
                kernels++;
            }
            // the source terms read lamF^s and the ghost-adjoint terms, which the
            // adjoint step and the probe residuals do not write: they run on the
            // side stream beside them, joined before the next ghost pass
            AdjSourceArgs sa{L, h->links, lam[la], gadj, {}, d_cells, ncell, s, d_out};
            std::copy(gadj_off, gadj_off + 6, sa.gadj_off);
            CK(cudaEventRecord(h->ev_fork, h->stream), "adjoint fork");
            CK(cudaStreamWaitEvent(h->side, h->ev_fork, 0), "adjoint fork");
            CK(launch_adj_source(sa, h->side), "adjoint source");
            CK(cudaEventRecord(h->ev_join, h->side), "adjoint join");
            kernels++;
            if (s > 0)
            {
                AdjStepArgs as{L, h->sa, lam[la], lam[la ^ 1], mom_of(s - 1 - cn), gadj, {}, adj_prefetch};
                std::copy(gadj_off, gadj_off + 6, as.gadj_off);
                CK(launch_adj_step(as, h->stream), "adjoint step");
                kernels++;
                la ^= 1;
                pa.resid = d_resid + (size_t)(s - 1) * np;
                CK(launch_adj_probe(lam[la], pa, h->stream), "adjoint probe");
                kernels++;
            }
            CK(cudaStreamWaitEvent(h->stream, h->ev_join, 0), "adjoint join");
        }
        return LBM_OK;
    };
    if (Tt < T)
    {
        st = reverse_segment(Tt, T, (int)cnT);
        if (st) return st;
    }
    for (int m = Mr - 1; m >= 0; --m)
    {
        const int O = m * K1, E = std::min(O + K1, Tt);
        const int N = (E - O + K2 - 1) / K2;
        CK(restore_g(outer, m), "restore");
        long long at = ckpt_pos(O);   // the current buffer holds G^at
        for (int n = 0; n < N; ++n)
        {
            const long long cn = ckpt_pos((long long)O + (long long)n * K2);
            for (; at < cn; ++at)
            {
                CK(source_ghost((int)at), "recompute");
                CK(collide((int)at, false), "recompute");
            }
            CK(save_g(inner, n), "checkpoint");
        }
        for (int n = N - 1; n >= 0; --n)
        {
            const int a0 = O + n * K2, a1 = std::min(a0 + K2, E);
            const int cn = (int)ckpt_pos(a0);
            CK(restore_g(inner, n), "restore");
            for (int s = cn; s < a1; ++s)
            {
                CK(stored_source_ghost(s, s - cn), "recompute");
                if (s + 1 < a1) CK(stored_collide(s - cn), "recompute");
            }
            st = reverse_segment(a0, a1, cn);
            if (st) return st;
        }
    }

    // ---- gradients: d L / d val_s = mu_s dt gain; d L / d pos = sum_s mass_s nu_s
    std::vector<double> out((size_t)T * 4);
    CK(cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
       "gradient download");
    CK(cudaStreamSynchronize(h->stream), "gradient download");
    h->launches += kernels;
    double gp[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < T; ++s)
    {
        for (int a = 0; a < 3; ++a) gp[a] += entries[s].mass * out[(size_t)s * 4 + 1 + a];
        if (grad_signal) grad_signal[s] = out[(size_t)s * 4] * h->dt * src.s.gain;
    }
    for (int s = 0; s < T; ++s)
        if (!std::isfinite(out[(size_t)s * 4])) return h->fail(LBM_ERR_NAN, "non-finite adjoint");
    if (grad_pos) std::copy(gp, gp + 3, grad_pos);
    if (predicted) std::copy(pred.begin(), pred.end(), predicted);
    *loss = Lsum;
    return rest_state(h);
}

// ---------------------------------------------------------------- z-slabs

namespace {

// side 0: the cut below the slab (toward slab_k0 - 1), side 1: the cut above it.
bool has_cut(const lbm_handle* h, int side)
{
    return h->slab && h->lcfg.face_bc[side ? LBM_FACE_ZHI : LBM_FACE_ZLO] == kBcCut;
}

int slab_msg_check(lbm_handle* h, int side, const void* msg)
{
    int st = check_ready(h);
    if (st) return st;
    if (side != 0 && side != 1) return h->fail(LBM_ERR_INVALID_ARGUMENT, "side is 0 (below) or 1 (above)");
    if (!has_cut(h, side)) return h->fail(LBM_ERR_STATE, "this z-slab has no cut on that side");
    if (!msg || ((uintptr_t)msg & 15u)) return h->fail(LBM_ERR_INVALID_ARGUMENT, "message buffer: 16-byte aligned device memory");
    return LBM_OK;
}

// pack: the plane next to the cut of `side` (plane 1 below, nz above), its
// directions toward the neighbour; unpack: the halo plane of that side, the
// neighbour's directions toward this slab.
cudaError_t slab_msg(lbm_handle* h, bool pack, int side, void* msg)
{
    const Layout& L = h->L;
    const int k = pack ? (side ? L.nz : 1) : (side ? L.nz + 1 : 0);
    const int up = pack ? side : 1 - side;
    return launch_slab_msg(pack, h->f[h->cur], h->xf.xgh, msg, L, k, up, h->storage == LBM_STORE_F16 ? 2 : 4,
                           h->stream);
}

int slab_buffers(lbm_handle* h)
{
    if (h->slab_buf) return LBM_OK;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    h->slab_msg_bytes = (size_t)(slab_message_bytes(h->L) + 255) / 256 * 256;
    CK(cudaMalloc(&h->slab_buf, 4 * h->slab_msg_bytes), "slab message buffers");
    CK(cudaEventCreateWithFlags(&h->ev_packed, cudaEventDisableTiming), "slab events");
    CK(cudaEventCreateWithFlags(&h->ev_read, cudaEventDisableTiming), "slab events");
    return LBM_OK;
}

char* slab_part(lbm_handle* h, int n) { return (char*)h->slab_buf + (size_t)n * h->slab_msg_bytes; }

}  // namespace

extern "C" long lbm_slab_message_bytes(lbm_handle* h)
{
    if (check_ready(h)) return 0;
    return h->slab ? (long)slab_message_bytes(h->L) : 0;
}

extern "C" int lbm_slab_pack(lbm_handle* h, int side, void* msg)
{
    int st = slab_msg_check(h, side, msg);
    if (st) return st;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    CK(slab_msg(h, true, side, msg), "slab pack");
    h->launches++;
    return LBM_OK;
}

extern "C" int lbm_slab_unpack(lbm_handle* h, int side, const void* msg)
{
    int st = slab_msg_check(h, side, msg);
    if (st) return st;
    CK(cudaSetDevice(h->device), "cudaSetDevice");
    CK(slab_msg(h, false, side, const_cast<void*>(msg)), "slab unpack");
    h->launches++;
    return LBM_OK;
}

extern "C" int lbm_slab_exchange(lbm_handle* lo, lbm_handle* hi)
{
    NvtxRange range("lbm_slab_exchange");
    if (!lo || !hi || lo == hi) return LBM_ERR_INVALID_ARGUMENT;
    int st = check_ready(lo);
    if (st) return st;
    st = check_ready(hi);
    if (st) return st;
    if (!lo->slab || !hi->slab) return lo->fail(LBM_ERR_STATE, "lbm_slab_exchange needs two z-slab handles");
    if (lo->cfg.slab_k0 + lo->cfg.slab_nz != hi->cfg.slab_k0)
        return lo->fail(LBM_ERR_INVALID_ARGUMENT, "the upper slab does not start where the lower one ends");
    if (lo->L.nx != hi->L.nx || lo->L.ny != hi->L.ny || lo->storage != hi->storage)
        return lo->fail(LBM_ERR_INVALID_ARGUMENT, "slabs of different grids");
    st = slab_buffers(lo);
    if (st) return st;
    st = slab_buffers(hi);
    if (st) return st;
    const size_t bytes = (size_t)slab_message_bytes(lo->L);
    // Only the populations that cross the cut travel: lower's top plane, ez = +1
    // (send part 1), into upper's halo plane 0; upper's bottom plane, ez = -1
    // (send part 0), into lower's halo plane nz + 1.  Each side packs on its own
    // stream after its halo fill; the receiver waits for that, copies the
    // message to its own GPU when the handles live on different ones, and
    // unpacks on its stream; each sender then waits until the receiver has
    // read its message before it packs the next one.
    const auto receive = [&](lbm_handle* to, int to_side, lbm_handle* from, int from_part) -> cudaError_t {
        cudaError_t e = cudaSetDevice(to->device);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(to->stream, from->ev_packed, 0);
        const void* src = slab_part(from, from_part);
        if (e == cudaSuccess && to->device != from->device)
        {
            e = cudaMemcpyPeerAsync(slab_part(to, 2 + to_side), to->device, src, from->device, bytes, to->stream);
            src = slab_part(to, 2 + to_side);
        }
        if (e == cudaSuccess) e = slab_msg(to, false, to_side, const_cast<void*>(src));
        if (e == cudaSuccess) e = cudaEventRecord(to->ev_read, to->stream);
        return e;
    };
    cudaError_t e = cudaSetDevice(lo->device);
    if (e == cudaSuccess) e = slab_msg(lo, true, 1, slab_part(lo, 1));
    if (e == cudaSuccess) e = cudaEventRecord(lo->ev_packed, lo->stream);
    if (e == cudaSuccess) e = cudaSetDevice(hi->device);
    if (e == cudaSuccess) e = slab_msg(hi, true, 0, slab_part(hi, 0));
    if (e == cudaSuccess) e = cudaEventRecord(hi->ev_packed, hi->stream);
    if (e == cudaSuccess) e = receive(hi, 0, lo, 1);
    if (e == cudaSuccess) e = receive(lo, 1, hi, 0);
    // neither handle packs into a buffer the other one is still reading
    if (e == cudaSuccess) e = cudaStreamWaitEvent(lo->stream, hi->ev_read, 0);
    if (e == cudaSuccess) e = cudaSetDevice(hi->device);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hi->stream, lo->ev_read, 0);
    cudaSetDevice(lo->device);
    if (e != cudaSuccess) return lo->cuda_fail(e, "slab exchange");
    lo->launches += 2;
    hi->launches += 2;
    return LBM_OK;
}
