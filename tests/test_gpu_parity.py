"""CUDA solver vs the FP64 oracle (and the reference fixtures), through the C-ABI.

Tolerances (stated per test): the device stores deviations from rest
equilibrium in FP32 (or scaled FP16) and collides in FP32, the oracle is the
reference's FP64 arithmetic.  The mask and all integer indexing are compared
bit for bit.
"""
import os

import numpy as np
import pytest

import nlos_lbm
import oracle
import scenarios
from nlos_lbm import abi
from scenarios import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# probe relative-L2 error vs the FP64 oracle, FP32 deviation storage (measured <= 3e-6)
FP32_PROBE_TOL = 1e-5
# largest population deviation error, relative to the largest deviation
FP32_STATE_TOL = 1e-4
# FP16 deviation storage with scale 1/amplitude: the 1e-3 probe target
FP16_PROBE_TOL = 1e-3

SCENARIOS = ["ref06_box", "ref08_moving", "scatter_small", "lloyd_small", "city_small"]


def deviation(f, dims_halo):
    nx, ny, nz = dims_halo
    a = f.reshape(nz, ny, nx, 19)[1:-1, 1:-1, 1:-1] - np.array(abi.W)
    return a


@pytest.mark.parametrize("name", SCENARIOS)
def test_fp32_matches_oracle(name, gpu):
    sc = scenarios.scenario(name)
    g, o = scenarios.build_pair(sc)
    assert g.dims_halo == o.dims_halo
    assert np.array_equal(g.get_mask(), o.get_mask())          # bit-exact voxelisation
    g.step(sc["steps"])
    o.step(sc["steps"])
    pg, po = g.get_probes(), o.get_probes()
    assert pg.shape == po.shape == (sc["steps"], len(sc["probes"]))
    assert np.max(np.abs(po)) > 0
    assert rel_l2(pg, po) <= FP32_PROBE_TOL, rel_l2(pg, po)
    dg, do = deviation(g.get_f(), g.dims_halo), deviation(o.get_f(), o.dims_halo)
    assert np.max(np.abs(dg - do)) <= FP32_STATE_TOL * np.max(np.abs(do))


@pytest.mark.parametrize("name", ["ref06_box", "ref08_moving", "ref06_empty"])
def test_fp32_matches_reference_fixture(name, gpu):
    from golden.make_golden import scenario_for

    sc = scenario_for(name)
    gold = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    assert np.array_equal(np.packbits(g.get_mask()), gold["mask_bits"])
    g.step(int(gold["steps"]))
    assert rel_l2(g.get_probes(), gold["probes"]) <= FP32_PROBE_TOL


@pytest.mark.parametrize("fixture", ["oracle_scatter_2000", "oracle_lloyd_6000", "oracle_city256_4000"])
def test_full_size_workload_matches_oracle_series(fixture, gpu):
    """The full-size 128^3 scattering box (2000 steps) and 256x128x128 Lloyd's
    mirror (6000 steps) benchmark workloads, and the 256x256x128 city patch
    with the 1024x1024x256 city's physics over its 4000 steps, FP32 and FP16
    storage (the workload's scale, 100/amplitude), against the FP64 oracle's
    series (tests/golden/make_oracle_series.py)."""
    from nlos_lbm import workloads

    path = os.path.join(GOLDEN, fixture + ".npz")
    if not os.path.exists(path):
        pytest.skip("oracle series not generated")
    gold = np.load(path)
    name, steps = fixture.split("_")[1], int(gold["steps"])
    for storage, tol in ((abi.LBM_STORE_F32, FP32_PROBE_TOL), (abi.LBM_STORE_F16, FP16_PROBE_TOL)):
        w = workloads.build(name, storage=storage)
        g = nlos_lbm.Solver(w["cfg"], w["sources"], w["probes"], triangles=w["triangles"])
        assert g.dims_halo == tuple(gold["dims_halo"])
        g.step(steps)
        err = rel_l2(g.get_probes(), gold["probes"])
        assert err <= tol, (name, storage, err)
        g.close()


@pytest.mark.parametrize("name", ["scatter_small", "lloyd_small", "city_small"])
def test_fp16_storage_matches_oracle(name, gpu):
    amp = {"scatter_small": 1e-3, "lloyd_small": 5e-4, "city_small": 1e-3}[name]
    sc = scenarios.scenario(name, storage=abi.LBM_STORE_F16, f16_scale=1.0 / amp)
    g, o = scenarios.build_pair(sc)
    g.step(sc["steps"])
    o.step(sc["steps"])
    assert rel_l2(g.get_probes(), o.get_probes()) <= FP16_PROBE_TOL, rel_l2(g.get_probes(), o.get_probes())


def test_standalone_calls_equal_batched_steps(gpu):
    """apply_source/exchange_halos/step_collision_bgk/record_probes one by one
    (the reference's call sequence, 06:1079-1092) equals lbm_step bit for bit."""
    sc = scenarios.scenario("ref08_moving")
    a = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    b = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    n = 37
    for s in range(n):
        a.apply_source(s * a.dt)
        a.exchange_halos()
        a.step_collision_bgk()
        a.record_probes()
    b.step(n)
    assert np.array_equal(a.get_probes(), b.get_probes())
    assert np.array_equal(a.get_f(), b.get_f())


def test_graphs_equal_direct_launches(gpu):
    sc = scenarios.scenario("city_small")
    cfg2 = scenarios.scenario("city_small")["cfg"]
    cfg2.use_graphs = 0
    a = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    b = nlos_lbm.Solver(cfg2, sc["sources"], sc["probes"], triangles=sc["triangles"])
    for chunk in (1, 6, 33):
        a.step(chunk)
        b.step(chunk)
    assert np.array_equal(a.get_probes(), b.get_probes())
    assert np.array_equal(a.get_f(), b.get_f())


def test_run_matches_reference_step_count(gpu):
    """run(T, Frames) takes round(T/dt)+1 steps (06:1066-1077)."""
    sc = scenarios.scenario("ref06_box")
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    o = oracle.OracleSolver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    T = 0.05
    g.run(T, 2)
    n = int(round(T / g.dt)) + 1
    assert g.step_count == n
    o.step(n)
    assert rel_l2(g.get_probes(), o.get_probes()) <= FP32_PROBE_TOL


def test_rest_state_is_exact(gpu):
    """No source: deviations stay exactly zero (the rest state is a fixed point)."""
    sc = scenarios.scenario("city_small")
    g = nlos_lbm.Solver(sc["cfg"], [], sc["probes"], triangles=sc["triangles"])
    g.step(7)
    assert np.all(g.get_probes() == 0.0)
    assert np.array_equal(deviation(g.get_f(), g.dims_halo), np.zeros_like(deviation(g.get_f(), g.dims_halo)))


def test_closed_box_conserves_mass(gpu):
    cfg = scenarios.lattice_config(40, 36, 30, 0.6, face_bc=(abi.LBM_BC_WALL,) * 6, sponge_faces=0)
    tris = oracle.box_triangles([(10, 10, 0, 20, 18, 12)])
    g = nlos_lbm.Solver(cfg, [], None, triangles=tris)
    o = oracle.OracleSolver(cfg, [], None, triangles=tris)
    nx, ny, nz = g.dims_halo
    f = o.get_f().reshape(nz, ny, nx, 19)
    rng = np.random.default_rng(3)
    f[1:-1, 1:-1, 1:-1] += 1e-3 * rng.standard_normal(f[1:-1, 1:-1, 1:-1].shape) * np.array(abi.W)
    g.set_f(f.ravel())
    o.set_f(f.ravel())
    # fluid mass only: a SOLID cell copies what it pulls (06:933-938)
    fluid = (g.get_mask().reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1] == 0)[..., None]
    d0 = deviation(f.ravel(), g.dims_halo)
    m0 = (d0 * fluid).sum()
    g.step(60)
    o.step(60)
    dg = deviation(g.get_f(), g.dims_halo)
    assert abs((dg * fluid).sum() - m0) <= 1e-5 * np.abs(d0 * fluid).sum()
    do = deviation(o.get_f(), o.dims_halo)
    assert np.max(np.abs(dg - do)) <= FP32_STATE_TOL * np.max(np.abs(do))


def test_probe_flags_and_solid_probe(gpu):
    """Probe outside the grid: not owned, NaN series; probe in a SOLID cell:
    warning status and rho-1 = 0 (06:415-437, 06:936)."""
    sc = scenarios.scenario("ref06_box")
    probes = np.vstack([sc["probes"], [[15.5, 13.5, 3.5], [-5.0, 3.0, 3.0]]])   # inside box 1; outside x
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], probes, triangles=sc["triangles"])
    assert abi.LBM_WARN_PROBE_IN_SOLID in g.warnings
    owned, solid = g.probe_info()
    assert list(owned) == [True] * 5 + [False]
    nx, ny, nz = g.dims_halo
    m = g.get_mask().reshape(nz, ny, nx)
    ijk = np.floor(probes[:5]).astype(int) + 1
    expect = [bool(m[k, j, i]) for i, j, k in ijk]
    assert expect[4] and list(solid) == expect + [False]
    g.step(40)
    p = g.get_probes()
    assert np.all(p[:, np.array(expect + [False])] == 0.0) and np.all(np.isnan(p[:, 5]))
    assert np.max(np.abs(p[:, 1])) > 0
    e = g.get_probe_energy()
    np.testing.assert_allclose(e[:5], (p[:, :5] ** 2).sum(0), rtol=1e-12)


def test_rho_field_matches_probes(gpu):
    sc = scenarios.scenario("lloyd_small")
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(90)
    rho = g.get_rho()
    p = g.get_probes()[-1]
    idx = np.floor(sc["probes"]).astype(int)
    np.testing.assert_array_equal(rho[idx[:, 2], idx[:, 1], idx[:, 0]].astype(np.float64), p.astype(np.float32))


def test_set_f_get_f_round_trip(gpu):
    sc = scenarios.scenario("scatter_small")
    g = nlos_lbm.Solver(sc["cfg"], [], None, triangles=sc["triangles"])
    nx, ny, nz = g.dims_halo
    rng = np.random.default_rng(5)
    f = (np.tile(np.array(abi.W), nx * ny * nz) * (1 + 1e-3 * rng.standard_normal(nx * ny * nz * 19)))
    g.set_f(f)
    back = g.get_f()
    dev_in = f - np.tile(np.array(abi.W), nx * ny * nz)
    dev_out = back - np.tile(np.array(abi.W), nx * ny * nz)
    np.testing.assert_allclose(dev_out, dev_in.astype(np.float32).astype(np.float64), rtol=0, atol=1e-12)


def translation_case(n3, offset, storage=abi.LBM_STORE_F32):
    """Point source and probes at fixed offsets from the grid centre, no sponge,
    rest halos: until a wave reaches a boundary the result cannot depend on
    the grid size."""
    nx, ny, nz = n3
    cfg = scenarios.lattice_config(nx, ny, nz, 0.51, face_bc=(abi.LBM_BC_REST,) * 6, sponge_faces=0,
                                   storage=storage, f16_scale=1000.0)
    cx, cy, cz = offset
    src = abi.reference_source(sx=cx + 0.5, sy=cy + 0.5, sz=cz + 0.5, ex=cx + 0.5, ey=cy + 0.5, ez=cz + 0.5,
                               amp=1e-3, freq=1 / 40.0, t0=40.0, waveform=abi.LBM_WAVE_RICKER)
    probes = np.array([[cx + 0.5 + d[0], cy + 0.5 + d[1], cz + 0.5 + d[2]]
                       for d in [(10, 0, 0), (0, -12, 3), (-7, 7, -7), (3, 2, 14)]])
    return cfg, [src], probes


@pytest.mark.parametrize("storage", [abi.LBM_STORE_F32, abi.LBM_STORE_F16])
def test_full_size_grid_translation_invariance(storage, gpu):
    """The 1024x1024x256 city-size grid gives bit-identical early-time probe
    series to a 48^3 grid around the same source (no cell or index of the
    large grid is mishandled), and the 48^3 run matches the oracle."""
    steps = 20   # the nearest small-grid boundary is 24 cells away
    big = translation_case((1024, 1024, 256), (700, 300, 130), storage)
    small = translation_case((48, 48, 48), (24, 24, 24), storage)
    gb = nlos_lbm.Solver(*big)
    gs = nlos_lbm.Solver(*small)
    gb.step(steps)
    gs.step(steps)
    assert np.array_equal(gb.get_probes(), gs.get_probes())
    if storage == abi.LBM_STORE_F32:
        o = oracle.OracleSolver(*small)
        o.step(steps)
        assert rel_l2(gs.get_probes(), o.get_probes()) <= FP32_PROBE_TOL
