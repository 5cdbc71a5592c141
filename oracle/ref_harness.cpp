/*
 * Include harness around the UNMODIFIED reference solver -- TEST INFRASTRUCTURE.
 *
 * Built by oracle/Makefile into oracle/_ref/libref06.so (from
 * 06_transient_localization_dx1.cpp, Gaussian-pulse source) and
 * oracle/_ref/libref08.so (from 08_city_scale_uav.cpp, moving sine source).
 * The reference file is #included where it lies; its `main` is renamed and its
 * private members are made reachable so the harness can read f_curr, rho and
 * mask after the public stepping methods run.  MPI comes from the single-rank
 * shim in oracle/mpi_shim/mpi.h.
 *
 * The harness calls the reference's own public methods in the order of
 * LBMSolver::run (06:1077-1092): apply_source(t) -> exchange_halos() ->
 * step_collision_bgk() -> probe record, with t = s * dt.  VTK output
 * (06:1094-1097) is skipped.
 *
 * Only tests/, bench.py's reference arm and the fixture generator load this.
 */
#include <mpi.h>
#include <omp.h>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define main reference_main
#define private public
#include REF_SOURCE
#undef private
#undef main

struct ref_params
{
    double x_min, x_max, y_min, y_max, z_min, z_max, dx;
    double tau;
    int use_geometry;
    int use_nscbc;
    const char* stl_file;
    double stl_sx, stl_sy, stl_sz;
    double d_sx, d_sy, d_sz, d_ex, d_ey, d_ez, d_speed, d_amp, d_freq;
    int n_probes;
    const double* probe_xyz;  // n_probes * 3
};

struct RefHandle
{
    LBMSolver s;
    std::vector<size_t> probe_idx;   // local index of owned probes (-1 if not owned)
    std::vector<std::vector<double>> series;
    int nx_t = 0, ny_t = 0, nz_t = 0;
};

extern "C" {

void* ref_create(const ref_params* p)
{
    auto* h = new RefHandle();
    LBMSolver& s = h->s;
    s.X_MIN = p->x_min; s.X_MAX = p->x_max;
    s.Y_MIN = p->y_min; s.Y_MAX = p->y_max;
    s.Z_MIN = p->z_min; s.Z_MAX = p->z_max;
    s.DX = p->dx;
    s.tau = p->tau;
    s.use_geometry = p->use_geometry != 0;
    s.use_nscbc = p->use_nscbc != 0;
    s.stl_file = p->stl_file ? p->stl_file : "";
    s.stl_sx = p->stl_sx; s.stl_sy = p->stl_sy; s.stl_sz = p->stl_sz;
    s.drone.sx = p->d_sx; s.drone.sy = p->d_sy; s.drone.sz = p->d_sz;
    s.drone.ex = p->d_ex; s.drone.ey = p->d_ey; s.drone.ez = p->d_ez;
    s.drone.speed = p->d_speed; s.drone.amp = p->d_amp; s.drone.freq = p->d_freq;

    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    s.init(0, nullptr);
    std::cout.rdbuf(old);

    h->nx_t = s.nx_t; h->ny_t = s.ny_t; h->nz_t = s.nz_t;
    const double dxp = s.units.dx_phys;
    for (int i = 0; i < p->n_probes; ++i)
    {
        const double* xyz = p->probe_xyz + 3 * i;
        // Same owner/index rule as LBMSolver::init (06:415-437).
        int gi = (int)std::floor((xyz[0] - s.X_MIN) / dxp);
        int gj = (int)std::floor((xyz[1] - s.Y_MIN) / dxp);
        int gk = (int)std::floor((xyz[2] - s.Z_MIN) / dxp);
        size_t idx = (size_t)-1;
        if (gi >= 0 && gi < s.nx && gj >= 0 && gj < s.ny && gk >= 0 && gk < s.nz)
            idx = loc_index(gi + 1, gj + 1, gk + 1, s.nx_t, s.ny_t);
        h->probe_idx.push_back(idx);
    }
    h->series.assign(p->n_probes, {});
    return h;
}

void ref_destroy(void* hp) { delete (RefHandle*)hp; }

void ref_dims(void* hp, int* out)
{
    auto* h = (RefHandle*)hp;
    out[0] = h->nx_t; out[1] = h->ny_t; out[2] = h->nz_t;
}

double ref_dt(void* hp) { return ((RefHandle*)hp)->s.units.get_dt_phys(); }

void ref_set_threads(int n) { omp_set_num_threads(n); }

void ref_apply_source(void* hp, double t) { ((RefHandle*)hp)->s.apply_source(t); }
void ref_exchange_halos(void* hp) { ((RefHandle*)hp)->s.exchange_halos(); }
void ref_step_collision_bgk(void* hp) { ((RefHandle*)hp)->s.step_collision_bgk(); }

void ref_record_probes(void* hp)
{
    auto* h = (RefHandle*)hp;
    for (size_t p = 0; p < h->probe_idx.size(); ++p)
        if (h->probe_idx[p] != (size_t)-1) h->series[p].push_back(h->s.rho[h->probe_idx[p]] - 1.0);
}

/* One full reference time step per s in [s0, s0+n), exactly the body of
 * LBMSolver::run (06:1079-1092) without VTK output. */
void ref_run_steps(void* hp, int s0, int n)
{
    auto* h = (RefHandle*)hp;
    const double dt = h->s.units.get_dt_phys();
    for (int s = s0; s < s0 + n; ++s)
    {
        const double t = s * dt;
        h->s.apply_source(t);
        h->s.exchange_halos();
        h->s.step_collision_bgk();
        ref_record_probes(hp);
    }
}

void ref_get_f(void* hp, double* out)
{
    auto* h = (RefHandle*)hp;
    std::memcpy(out, h->s.f_curr.data(), h->s.f_curr.size() * sizeof(double));
}

void ref_set_f(void* hp, const double* in)
{
    auto* h = (RefHandle*)hp;
    std::memcpy(h->s.f_curr.data(), in, h->s.f_curr.size() * sizeof(double));
}

void ref_get_rho(void* hp, double* out)
{
    auto* h = (RefHandle*)hp;
    std::memcpy(out, h->s.rho.data(), h->s.rho.size() * sizeof(double));
}

void ref_get_mask(void* hp, uint8_t* out)
{
    auto* h = (RefHandle*)hp;
    std::memcpy(out, h->s.mask.data(), h->s.mask.size());
}

void ref_get_sponge(void* hp, double* out)
{
    auto* h = (RefHandle*)hp;
    std::memcpy(out, h->s.sponge_sigma.data(), h->s.sponge_sigma.size() * sizeof(double));
}

/* Probe series, layout [step][probe]; unowned probes are NaN. */
int ref_get_probes(void* hp, double* out, long capacity)
{
    auto* h = (RefHandle*)hp;
    const size_t np = h->series.size();
    size_t steps = 0;
    for (auto& v : h->series) steps = std::max(steps, v.size());
    if ((long)(steps * np) > capacity) return -1;
    for (size_t s = 0; s < steps; ++s)
        for (size_t p = 0; p < np; ++p)
            out[s * np + p] = s < h->series[p].size() ? h->series[p][s] : NAN;
    return (int)steps;
}

}  // extern "C"
