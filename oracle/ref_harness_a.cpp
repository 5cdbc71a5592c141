/*
 * Harness for the reference's family-A programs -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiles one unmodified family-A program (01_acoustic_scattering.cpp with
 * REF_PROG=1, 02_lloyds_mirror.cpp with REF_PROG=2, 03_doppler_effect.cpp
 * with REF_PROG=3, 04_hpc_scalability.cpp with REF_PROG=4) where it lies, with the
 * single-rank MPI shim, and exposes its Solver through a small C interface so
 * tests can run it on reduced domains and compare the oracle's family-A
 * restatement with it.  Each reference time step is exchange_halos() then
 * step(): 02 passes the physical time s*dt (02:543-546), 03 the step index s
 * (03:540-541); 01's step is step_pull() (01:527-528); 04's is
 * apply_source(s*dt, dt), exchange_halos(), step_pull() (04:383-389).
 * Nothing in the product library links this file.
 */
#include <mpi.h>
#include <omp.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <vector>

#define main reference_main
#include REF_SOURCE
#undef main
#if REF_PROG == 4
using Solver = LBM;   // 04 names its solver LBM
#endif

struct refa_params
{
    double x_min, x_max, y_min, y_max, z_min, z_max, dx;   // domain (01, 02); 03 takes nx = (x_max-x_min)/dx etc.
    double amp;                 // source amplitude (02, 03, 04); 01: initial pulse amplitude (01:67)
    double b_param;             // 02, 04: source width parameter (02:181, 04:67; <= 0: keep 04's)
    double omega;               // 02, 04: angular frequency, rad per physical second (<= 0: keep 02:126, 04:68)
    double Ma;                  // 03: background Mach number (03:55)
    double tau_bulk, tau_sponge_max;   // 03 (03:61-62)
    int sponge_width;           // 03 (03:63)
    double omega_lb;            // 03: angular frequency per step (<= 0: keep 03:121)
};

struct RefAHandle
{
    Solver s;
    long step = 0;
};

extern "C" {

void* refa_create(const refa_params* p)
{
    auto* h = new RefAHandle();
    Solver& s = h->s;
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
#if REF_PROG == 1
    s.X_MIN = p->x_min; s.X_MAX = p->x_max;
    s.Y_MIN = p->y_min; s.Y_MAX = p->y_max;
    s.Z_MIN = p->z_min; s.Z_MAX = p->z_max;
    s.units.dx_phys = p->dx;
    s.pulse_amp_lbm = p->amp;
    s.setup_mpi(0, nullptr);
#elif REF_PROG == 4
    s.X_MIN = p->x_min; s.X_MAX = p->x_max;
    s.Y_MIN = p->y_min; s.Y_MAX = p->y_max;
    s.Z_MIN = p->z_min; s.Z_MAX = p->z_max;
    s.units.dx_phys = p->dx;
    s.Amp = p->amp;
    if (p->b_param > 0) s.b_param = p->b_param;
    if (p->omega > 0) s.omega = p->omega;
    s.setup_mpi(0, nullptr);
#elif REF_PROG == 2
    s.X_MIN = p->x_min; s.X_MAX = p->x_max;
    s.Y_MIN = p->y_min; s.Y_MAX = p->y_max;
    s.Z_MIN = p->z_min; s.Z_MAX = p->z_max;
    s.units.dx_phys = p->dx;
    s.amp = p->amp;
    s.b_param = p->b_param;
    s.setup_mpi(0, nullptr);
    if (p->omega > 0) s.omega = p->omega;
#else
    s.NXg = (int)((p->x_max - p->x_min) / p->dx + 0.5);
    s.NYg = (int)((p->y_max - p->y_min) / p->dx + 0.5);
    s.NZg = (int)((p->z_max - p->z_min) / p->dx + 0.5);
    s.units.dx_phys = p->dx;
    s.Ma = p->Ma;
    s.amp = p->amp;
    s.tau_bulk = p->tau_bulk;
    s.tau_sponge_max = p->tau_sponge_max;
    s.sponge_width = p->sponge_width;
    s.setup_mpi(0, nullptr);
    if (p->omega_lb > 0) s.omega_lb = p->omega_lb;
#endif
    s.init_physics();
    std::cout.rdbuf(old);
    return h;
}

void refa_destroy(void* hp) { delete (RefAHandle*)hp; }
void refa_set_threads(int n) { omp_set_num_threads(n); }

void refa_dims(void* hp, int* n3_halo)
{
    auto& s = ((RefAHandle*)hp)->s;
    n3_halo[0] = s.nx_t; n3_halo[1] = s.ny_t; n3_halo[2] = s.nz_t;
}

double refa_dt(void* hp) { return ((RefAHandle*)hp)->s.units.get_dt_phys(); }

void refa_step(void* hp, int n)
{
    auto* h = (RefAHandle*)hp;
    Solver& s = h->s;
    const double dt = s.units.get_dt_phys();
    for (int i = 0; i < n; ++i, ++h->step)
    {
#if REF_PROG == 4
        s.apply_source(h->step * dt, dt);
#endif
        s.exchange_halos();
#if REF_PROG == 1 || REF_PROG == 4
        (void)dt;
        s.step_pull();
#elif REF_PROG == 2
        s.step(h->step * dt);
#else
        (void)dt;
        s.step((int)h->step);
#endif
    }
}

void refa_get_rho(void* hp, double* out)
{
    auto& s = ((RefAHandle*)hp)->s;
    std::memcpy(out, s.rho.data(), s.rho.size() * sizeof(double));
}

void refa_get_f(void* hp, double* out)
{
    auto& s = ((RefAHandle*)hp)->s;
    std::memcpy(out, s.f_curr.data(), s.f_curr.size() * sizeof(double));
}

void refa_get_tau(void* hp, double* out)
{
    auto& s = ((RefAHandle*)hp)->s;
#if REF_PROG == 1
    std::fill(out, out + s.rho.size(), 0.505);   // 01:305, one tau everywhere
#elif REF_PROG == 4
    std::fill(out, out + s.rho.size(), 0.51);    // 04:301
#else
    std::memcpy(out, s.tau_field.data(), s.tau_field.size() * sizeof(double));
#endif
}

void refa_get_source(void* hp, double* out)
{
    auto& s = ((RefAHandle*)hp)->s;
#if REF_PROG == 1 || REF_PROG == 4
    std::fill(out, out + s.rho.size(), 0.0);   // 01 has an initial pulse; 04 computes its source per step
#else
    std::memcpy(out, s.source_spatial.data(), s.source_spatial.size() * sizeof(double));
#endif
}

// 01's and 04's destination-blend sponge (01:207-225, 04:177-209); 0 for 02 and 03 (their sponge
// is a tau ramp)
void refa_get_sponge(void* hp, double* out)
{
    auto& s = ((RefAHandle*)hp)->s;
#if REF_PROG == 1 || REF_PROG == 4
    std::memcpy(out, s.sponge_sigma.data(), s.sponge_sigma.size() * sizeof(double));
#else
    std::fill(out, out + s.rho.size(), 0.0);
#endif
}

void refa_get_mask(void* hp, unsigned char* out)
{
    auto& s = ((RefAHandle*)hp)->s;
    const size_t n = (size_t)s.nx_t * s.ny_t * s.nz_t;
#if REF_PROG == 1 || REF_PROG == 2 || REF_PROG == 4
    std::memcpy(out, s.mask.data(), n);
#else
    std::memset(out, 0, n);   // 03 has no solid cells
#endif
}

}  // extern "C"
