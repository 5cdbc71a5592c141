"""Generates tests/golden/*.npz from the UNMODIFIED reference solver.

Run from the repository root where the reference sources are available:

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture runs one reference-native scenario of tests/scenarios.py through
oracle/_ref/libref06.so or libref08.so (the reference's own apply_source /
exchange_halos / step_collision_bgk, 06:1077-1092) and stores the probe
series, the voxelised mask, a window of the final populations and two FP64
checksums of the whole population array.  The family-A fixtures (lloyd_a,
doppler_a, scattering_a, hpc_a) run 02_lloyds_mirror.cpp / 03_doppler_effect.cpp /
01_acoustic_scattering.cpp / 04_hpc_scalability.cpp through oracle/_ref/libref02.so /
libref03.so / libref01.so / libref04.so (exchange_halos + step, 02:543-546,
03:540-541, 01:527-528; 04 with apply_source first, 04:383-389) and store the
final density field.  `python tests/golden/make_golden.py NAME ...`
regenerates only the named fixtures.  The fixtures pin the oracle (and,
within tolerance, the CUDA solver) to the reference on machines where the
reference itself is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200"))

import oracle  # noqa: E402
import scenarios  # noqa: E402

CASES = {
    # name: (reference program, scenario)
    "ref06_box": "06",
    "ref08_moving": "08",
    "ref06_empty": "06",
}


def scenario_for(name):
    if name == "ref06_empty":
        sc = scenarios.scenario("ref06_box")
        sc["triangles"] = None
        sc["cfg"].use_geometry = 0
        return sc
    return scenarios.scenario(name)


def checksums(f):
    w = np.random.default_rng(1234).standard_normal(f.size)
    return np.array([f.sum(), float(np.dot(f, w))])


def window(f, dims_halo):
    nx, ny, nz = dims_halo
    a = f.reshape(nz, ny, nx, 19)
    return np.ascontiguousarray(a[nz // 2, 2:18, 2:18, :])


def reference_run(name):
    sc = scenario_for(name)
    which = CASES[name]
    c = sc["cfg"]
    s = sc["sources"][0]
    stl = None
    if sc["triangles"] is not None:
        stl = os.path.join("/tmp", f"golden_{name}.stl")
        oracle.write_stl(stl, sc["triangles"])
    ref = oracle.RefSolver(which, (c.x_min, c.x_max), (c.y_min, c.y_max), (c.z_min, c.z_max), c.dx, c.tau,
                           (s.sx, s.sy, s.sz, s.ex, s.ey, s.ez, s.speed, s.amp, s.freq), probes=sc["probes"],
                           stl=stl, use_geometry=bool(c.use_geometry))
    ref.step(sc["steps"])
    f = ref.get_f()
    return dict(probes=ref.get_probes(), mask_bits=np.packbits(ref.get_mask()), f_window=window(f, ref.dims_halo),
                f_checksums=checksums(f), dims_halo=np.array(ref.dims_halo), steps=np.array(sc["steps"]))


FAMILY_A = ("lloyd_a", "doppler_a", "scattering_a", "hpc_a")


def reference_run_a(name):
    """A family-A program (01, 02, 03 or 04) on its reduced scenario: rho - 1 of every
    interior cell after the scenario's steps (SOLID cells as 0), its tau and
    source-weight fields and the mask."""
    sc = scenarios.family_a(name)
    ref = oracle.RefASolver(sc["ref"], **sc["ref_params"])
    ref.step(sc["steps"])
    nx, ny, nz = ref.dims_halo
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    rho = ref.get_rho().reshape(nz, ny, nx)[inner] - 1.0
    mask = ref.get_mask().reshape(nz, ny, nx)
    rho[mask[inner] == 1] = 0.0
    return dict(rho_minus_1=rho, mask_bits=np.packbits(mask), dims_halo=np.array(ref.dims_halo),
                steps=np.array(sc["steps"]), dt=np.array(ref.dt))


def main(names=()):
    oracle.build(ref=True)
    for name in CASES:
        if names and name not in names:
            continue
        out = reference_run(name)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, {k: v.shape for k, v in out.items()})
    for name in FAMILY_A:
        if names and name not in names:
            continue
        out = reference_run_a(name)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
