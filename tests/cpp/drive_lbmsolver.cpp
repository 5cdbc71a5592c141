// Scenario driver written against the LBMSolver interface (test input for
// tests/test_cpp_mirror.py): a 48 x 32 x 30 m box with dx = 1 m, the STL
// geometry given on the command line, a stationary Gaussian-pulse source
// and four probes, run for T = 79 dt (80 steps, frames at steps 0, 39, 78).
#include <cstdio>
#include <cstdlib>

#include "lbm_solver.hpp"

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: %s geometry.stl [fp16]\n", argv[0]);
        return 2;
    }
    nlos::LBMSolver s;
    s.DX = 1.0;
    s.stl_file = argv[1];
    s.X_MIN = 0.0; s.X_MAX = 48.0;
    s.Y_MIN = 0.0; s.Y_MAX = 32.0;
    s.Z_MIN = 0.0; s.Z_MAX = 30.0;
    s.probes.push_back({"A", 20.5, 16.5, 10.5});
    s.probes.push_back({"B", 30.5, 16.5, 20.5});
    s.probes.push_back({"C", 5.2, 3.3, 2.1});
    s.probes.push_back({"D", 44.0, 28.0, 25.0});
    s.drone.sx = s.drone.ex = 24.3;
    s.drone.sy = s.drone.ey = 16.2;
    s.drone.sz = s.drone.ez = 12.7;
    s.drone.speed = 0.0;
    s.drone.amp = 10.0;
    if (argc > 2)
    {
        s.storage = LBM_STORE_F16;
        s.f16_scale = 100.0;
    }
    s.init(argc, argv);
    const double T = 79 * s.dt();
    s.run(T, 2);
    return 0;
}
