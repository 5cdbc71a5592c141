// lbm_solver.hpp -- C++ mirror of the reference solver class over the C-ABI.
//
// nlos::LBMSolver has the public fields and methods of LBMSolver in
// 06_transient_localization_dx1.cpp:241-1122 (and its 08 sibling), so a
// scenario `main` written against the reference compiles against this header
// with the include and the class namespace changed.  The work runs on one
// B200 through liblbm_b200.so (include/nlos_lbm.h); this header only holds
// host glue.  Errors of the library are thrown as std::runtime_error; the
// warnings the reference prints (STL not loaded 06:409, probe inside a
// building 06:434) are printed the same way.
//
// Differences in what is written to disk: probe files use the reference's
// name and format (probe_<name>.txt, %.8e per line, 06:1106-1118); VTK frames
// use the reference's file names and header (output_mpi/flight_%05d.vtk,
// 06:1031-1053) with BINARY float32 data instead of ASCII.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "nlos_lbm.h"

namespace nlos {

// DroneSource (06:211-239): straight flight from (sx,sy,sz) to (ex,ey,ez).
struct DroneSource
{
    double sx = 0, sy = 0, sz = 0;
    double ex = 0, ey = 0, ez = 0;
    double speed = 0;
    double amp = 0;
    double freq = 0;
    double cx = 0, cy = 0, cz = 0;
};

class LBMSolver
{
public:
    // ---- public fields of the reference (06:244-268, 06:669) ----
    std::string stl_file;
    double stl_sx = 0.0, stl_sy = 0.0, stl_sz = 0.0;
    DroneSource drone;
    bool use_geometry = true;
    double X_MIN = 0.0, X_MAX = 1650.0;
    double Y_MIN = 0.0, Y_MAX = 1150.0;
    double Z_MIN = 0.0, Z_MAX = 250.0;
    double DX = 2.0;
    bool output_world_coords = true;
    struct Probe
    {
        std::string name;
        double x, y, z;
        int gi = 0, gj = 0, gk = 0;
        int li = 0, lj = 0, lk = 0;
        bool owned = false;
        std::vector<double> p_history;
    };
    std::vector<Probe> probes;
    double tau = 0.55;
    bool use_nscbc = true;

    // ---- knobs of this library (defaults reproduce the reference) ----
    int waveform = LBM_WAVE_GAUSS;   // LBM_WAVE_SINE reproduces 08_city_scale_uav.cpp
    int storage = LBM_STORE_F32;     // LBM_STORE_F16: deviations in FP16, scaled by f16_scale
    double f16_scale = 1.0;
    int device = 0;
    bool write_files = true;         // probe files and VTK frames in run()

    LBMSolver() = default;
    LBMSolver(const LBMSolver&) = delete;
    LBMSolver& operator=(const LBMSolver&) = delete;
    ~LBMSolver()
    {
        if (h_) lbm_destroy(h_);
    }

    // LBMSolver::init (06:299-450): grid, mask, sponge, rest state, probes.
    void init(int /*argc*/ = 0, char** /*argv*/ = nullptr)
    {
        lbm_config c;
        lbm_config_default(&c);
        c.x_min = X_MIN; c.x_max = X_MAX;
        c.y_min = Y_MIN; c.y_max = Y_MAX;
        c.z_min = Z_MIN; c.z_max = Z_MAX;
        c.dx = DX;
        c.tau = tau;
        c.use_geometry = use_geometry ? 1 : 0;
        if (!use_nscbc)
            for (int f = 0; f < 6; ++f)
                if (c.face_bc[f] == LBM_BC_NSCBC) c.face_bc[f] = LBM_BC_REST;
        c.storage = storage;
        c.f16_scale = f16_scale;
        c.device = device;
        if (h_) lbm_destroy(h_);
        h_ = nullptr;
        check(lbm_create(&c, &h_), "lbm_create");
        if (use_geometry)
        {
            const int st = lbm_set_geometry_stl(h_, stl_file.c_str(), 1.0, stl_sx, stl_sy, stl_sz);
            if (st == LBM_WARN_STL_NOT_LOADED) std::cout << "Warning: STL not loaded, using empty geometry.\n";
            else check(st, "lbm_set_geometry_stl");
        }
        lbm_source s;
        lbm_source_default(&s);
        s.sx = drone.sx; s.sy = drone.sy; s.sz = drone.sz;
        s.ex = drone.ex; s.ey = drone.ey; s.ez = drone.ez;
        s.speed = drone.speed;
        s.amp = drone.amp;
        s.freq = drone.freq;
        s.waveform = waveform;
        check(lbm_add_source(h_, &s), "lbm_add_source");
        std::vector<double> xyz;
        for (const auto& p : probes)
        {
            xyz.push_back(p.x);
            xyz.push_back(p.y);
            xyz.push_back(p.z);
        }
        if (!probes.empty()) check(lbm_set_probes(h_, xyz.data(), (int)probes.size()), "lbm_set_probes");
        const int st = lbm_init(h_);
        if (st < 0) check(st, "lbm_init");
        dt_ = lbm_get_dt(h_);
        int n3[3];
        check(lbm_get_dims(h_, n3, nullptr), "lbm_get_dims");
        NXg = n3[0]; NYg = n3[1]; NZg = n3[2];
        if (!probes.empty())
        {
            std::vector<int> owned(probes.size()), solid(probes.size());
            check(lbm_probe_info(h_, owned.data(), solid.data()), "lbm_probe_info");
            for (size_t p = 0; p < probes.size(); ++p)
            {
                Probe& pr = probes[p];
                pr.gi = (int)std::floor((pr.x - X_MIN) / DX);   // 06:417-419
                pr.gj = (int)std::floor((pr.y - Y_MIN) / DX);
                pr.gk = (int)std::floor((pr.z - Z_MIN) / DX);
                pr.owned = owned[p] != 0;
                pr.li = pr.gi + 1; pr.lj = pr.gj + 1; pr.lk = pr.gk + 1;
                pr.p_history.clear();
                if (solid[p]) std::cout << "WARNING: Probe " << pr.name << " is trapped inside SOLID building!\n";
            }
        }
        recorded_ = 0;
    }

    // The per-step members (06:576, 06:671, 06:906).
    void apply_source(double t) { check(lbm_apply_source(h_, t), "lbm_apply_source"); }
    void exchange_halos() { check(lbm_exchange_halos(h_), "lbm_exchange_halos"); }
    void step_collision_bgk() { check(lbm_step_collision_bgk(h_), "lbm_step_collision_bgk"); }
    // Probe record of the last step (06:1085-1092).
    void record_probes()
    {
        check(lbm_record_probes(h_), "lbm_record_probes");
        pull_probes();
    }

    // LBMSolver::write_vtk (06:975-1062): (float)(rho-1) on the whole grid.
    void write_vtk(int frame_id)
    {
        std::cout << "Write VTK frame " << frame_id << " ...\n";
        const size_t n = (size_t)NXg * NYg * NZg;
        std::vector<float> p(n);
        check(lbm_get_rho(h_, p.data(), (long)n), "lbm_get_rho");
        ::mkdir("output_mpi", 0755);
        char fn[64];
        std::snprintf(fn, sizeof fn, "output_mpi/flight_%05d.vtk", frame_id);
        std::ofstream f(fn, std::ios::binary);
        double ox = X_MIN, oy = Y_MIN, oz = Z_MIN;
        if (output_world_coords)
        {
            ox += -stl_sx;   // world_offset() (06:293-296)
            oy += -stl_sy;
            oz += -stl_sz;
        }
        f << "# vtk DataFile Version 3.0\nLBM Urban Acoustics V21\nBINARY\n";
        f << "DATASET STRUCTURED_POINTS\n";
        f << "DIMENSIONS " << NXg << " " << NYg << " " << NZg << "\n";
        f << "ORIGIN " << ox << " " << oy << " " << oz << "\n";
        f << "SPACING " << DX << " " << DX << " " << DX << "\n";
        f << "POINT_DATA " << n << "\n";
        f << "SCALARS PressureAmp float 1\nLOOKUP_TABLE default\n";
        for (float v : p)   // legacy VTK binary data are big-endian
        {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
            f.write(reinterpret_cast<const char*>(&u), 4);
        }
    }

    // LBMSolver::run (06:1064-1121): steps s = 0..round(T/dt) with a VTK frame
    // every total_steps/Frames steps, then one probe file per owned probe.
    void run(double T_total, int Frames)
    {
        const int total_steps = (int)std::round(T_total / dt_);
        const int out_interval = std::max(1, total_steps / std::max(Frames, 1));
        std::cout << "Run: T_total=" << T_total << " s, Frames=" << Frames << ", total_steps=" << total_steps
                  << ", out_interval=" << out_interval << "\n";
        int frame_id = 0;
        int s = 0;
        while (s <= total_steps)
        {
            // steps up to and including the next frame step run as one batch
            const int next_frame = ((s + out_interval - 1) / out_interval) * out_interval;
            const int last = std::min(total_steps, next_frame);
            check(lbm_step(h_, last - s + 1), "lbm_step");
            s = last + 1;
            if (last % out_interval == 0 && write_files) write_vtk(frame_id++);
            std::cout << "Step " << last << "/" << total_steps << "\r" << std::flush;
        }
        pull_probes();
        if (write_files)
            for (const auto& p : probes)
            {
                if (!p.owned) continue;
                std::ofstream out("probe_" + p.name + ".txt");
                for (double v : p.p_history) out << std::scientific << std::setprecision(8) << v << "\n";
                std::cout << "Rank 0 successfully wrote probe_" << p.name << ".txt (" << p.p_history.size()
                          << " steps)\n";
            }
        std::cout << "\nDone.\n";
    }

    double dt() const { return dt_; }
    lbm_handle* handle() { return h_; }
    int NXg = 0, NYg = 0, NZg = 0;

private:
    void check(int st, const char* what)
    {
        if (st < 0)
            throw std::runtime_error(std::string(what) + ": " + lbm_status_string(st) +
                                     (h_ ? std::string(" (") + lbm_last_error(h_) + ")" : std::string()));
    }
    // Appends the probe rows recorded since the last pull to p_history.
    void pull_probes()
    {
        if (probes.empty()) return;
        long rows = 0;
        check(lbm_get_probes(h_, nullptr, 0, &rows), "lbm_get_probes");
        std::vector<double> all((size_t)rows * probes.size());
        check(lbm_get_probes(h_, all.data(), (long)all.size(), &rows), "lbm_get_probes");
        for (long r = recorded_; r < rows; ++r)
            for (size_t p = 0; p < probes.size(); ++p)
                if (probes[p].owned) probes[p].p_history.push_back(all[(size_t)r * probes.size() + p]);
        recorded_ = rows;
    }

    lbm_handle* h_ = nullptr;
    double dt_ = 0.0;
    long recorded_ = 0;
};

}  // namespace nlos
