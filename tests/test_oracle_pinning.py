"""The FP64 oracle is pinned to the reference solver.

1. Against the committed fixtures (tests/golden/*.npz, made by
   make_golden.py from the unmodified reference): probes, mask, a population
   window and whole-array checksums must be bit-identical.
2. Against the live reference harness (oracle/_ref), when it was built here:
   the full population array, rho, sponge and mask, bit-identical.
"""
import os

import numpy as np
import pytest

import oracle
import scenarios
from golden.make_golden import CASES, checksums, scenario_for, window

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run_oracle(name):
    sc = scenario_for(name)
    o = oracle.OracleSolver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    o.step(sc["steps"])
    return o


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_fixture(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    o = run_oracle(name)
    assert tuple(g["dims_halo"]) == o.dims_halo
    assert np.array_equal(np.packbits(o.get_mask()), g["mask_bits"])
    np.testing.assert_array_equal(o.get_probes(), g["probes"])
    f = o.get_f()
    np.testing.assert_array_equal(window(f, o.dims_halo), g["f_window"])
    np.testing.assert_array_equal(checksums(f), g["f_checksums"])


@pytest.mark.skipif(not oracle.ref_available("06"), reason="reference harness not built here")
@pytest.mark.parametrize("with_geometry", [False, True])
def test_oracle_bit_identical_to_live_reference(with_geometry, tmp_path):
    sc = scenarios.scenario("ref06_box")
    c = sc["cfg"]
    stl = None
    if with_geometry:
        stl = str(tmp_path / "g.stl")
        oracle.write_stl(stl, sc["triangles"])
    else:
        c.use_geometry = 0
    s = sc["sources"][0]
    ref = oracle.RefSolver("06", (c.x_min, c.x_max), (c.y_min, c.y_max), (c.z_min, c.z_max), c.dx, c.tau,
                           (s.sx, s.sy, s.sz, s.ex, s.ey, s.ez, s.speed, s.amp, s.freq), probes=sc["probes"],
                           stl=stl, use_geometry=with_geometry)
    orc = oracle.OracleSolver(c, [s], sc["probes"], stl=stl)
    assert np.array_equal(ref.get_mask(), orc.get_mask())
    assert np.array_equal(ref.get_sponge(), orc.get_sponge())
    for chunk in (1, 9, 30):
        ref.step(chunk)
        orc.step(chunk)
        assert np.array_equal(ref.get_f(), orc.get_f())
        assert np.array_equal(ref.get_rho(), orc.get_rho())
    np.testing.assert_array_equal(ref.get_probes(), orc.get_probes())


@pytest.mark.skipif(not oracle.ref_available("08"), reason="reference harness not built here")
def test_oracle_bit_identical_to_live_reference_moving_sine(tmp_path):
    sc = scenarios.scenario("ref08_moving")
    c = sc["cfg"]
    stl = str(tmp_path / "g.stl")
    oracle.write_stl(stl, sc["triangles"])
    s = sc["sources"][0]
    ref = oracle.RefSolver("08", (c.x_min, c.x_max), (c.y_min, c.y_max), (c.z_min, c.z_max), c.dx, c.tau,
                           (s.sx, s.sy, s.sz, s.ex, s.ey, s.ez, s.speed, s.amp, s.freq), probes=sc["probes"], stl=stl)
    orc = oracle.OracleSolver(c, [s], sc["probes"], stl=stl)
    ref.step(sc["steps"])
    orc.step(sc["steps"])
    assert np.array_equal(ref.get_f(), orc.get_f())
    np.testing.assert_array_equal(ref.get_probes(), orc.get_probes())


@pytest.mark.skipif(not oracle.ref_available("06"), reason="reference harness not built here")
def test_oracle_use_nscbc_false_matches_reference(tmp_path):
    """use_nscbc = false (06:669) holds every halo at rest: the REST face type."""
    from nlos_lbm import abi

    sc = scenarios.scenario("ref06_box")
    c = sc["cfg"]
    c.use_geometry = 0
    for f in range(6):
        if c.face_bc[f] == abi.LBM_BC_NSCBC:
            c.face_bc[f] = abi.LBM_BC_REST
    s = sc["sources"][0]
    ref = oracle.RefSolver("06", (c.x_min, c.x_max), (c.y_min, c.y_max), (c.z_min, c.z_max), c.dx, c.tau,
                           (s.sx, s.sy, s.sz, s.ex, s.ey, s.ez, s.speed, s.amp, s.freq), probes=sc["probes"],
                           use_geometry=False, use_nscbc=False)
    orc = oracle.OracleSolver(c, [s], sc["probes"])
    ref.step(50)
    orc.step(50)
    assert np.array_equal(ref.get_f(), orc.get_f())


def test_oracle_rest_state_is_fixed_point():
    """feq(1, 0) is a BGK fixed point (06:958-964): no source, nothing moves.
    In the reference's FP64 f-form the weights do not sum to exactly 1, so the
    rest state holds to rounding (1e-15), not bit for bit."""
    sc = scenarios.scenario("scatter_small")
    o = oracle.OracleSolver(sc["cfg"], [], sc["probes"], triangles=sc["triangles"])
    f0 = o.get_f()
    o.step(5)
    f1 = o.get_f()
    nx, ny, nz = o.dims_halo
    a0 = f0.reshape(nz, ny, nx, 19)[1:-1, 1:-1, 1:-1]
    a1 = f1.reshape(nz, ny, nx, 19)[1:-1, 1:-1, 1:-1]
    assert np.max(np.abs(a0 - a1)) < 1e-15
    assert np.max(np.abs(o.get_probes())) < 1e-14


def test_oracle_closed_box_conserves_mass():
    """All faces WALL, no sponge, no source: sum f is conserved to rounding."""
    from nlos_lbm import abi

    cfg = scenarios.lattice_config(20, 18, 16, 0.6, face_bc=(abi.LBM_BC_WALL,) * 6, sponge_faces=0)
    o = oracle.OracleSolver(cfg, [], None)
    nx, ny, nz = o.dims_halo
    f = o.get_f().reshape(nz, ny, nx, 19)
    rng = np.random.default_rng(0)
    f[1:-1, 1:-1, 1:-1] += 1e-3 * rng.standard_normal(f[1:-1, 1:-1, 1:-1].shape) * np.array(oracle.abi.W)
    o.set_f(f.ravel())
    m0 = f[1:-1, 1:-1, 1:-1].sum()
    o.step(40)
    m1 = o.get_f().reshape(nz, ny, nx, 19)[1:-1, 1:-1, 1:-1].sum()
    assert abs(m1 - m0) < 1e-10 * abs(m0)
