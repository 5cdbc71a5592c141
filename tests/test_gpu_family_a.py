"""Scheme A (the reference's family-A programs 01-04) on the GPU, through the
C-ABI, against the FP64 oracle's family-A restatement (itself checked
against the unmodified 01/02/03 programs in tests/test_oracle_family_a.py
and the fixtures in tests/golden/).

Tolerances: FP32 deviation storage against FP64, probe (density) series
relative L2 <= 1e-5 and field max error <= 1e-5 of the field's largest
deviation, the FP32 bars of the scheme-B parity tests.
"""
import ctypes
import os

import numpy as np
import pytest

import scenarios
from nlos_lbm import LBMError, Solver, abi
from oracle import OracleSolver
from scenarios import rel_l2

pytestmark = pytest.mark.gpu

PROBE_TOL = 1e-5
FIELD_TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _solver(sc, **kw):
    g = Solver(sc["cfg"], sc["sources"], sc["probes"], mask=sc["mask"], blend_xy=sc.get("blend_xy"),
               field_xy=sc.get("field_xy"), **kw)
    if sc.get("rho0") is not None:
        g.set_density(sc["rho0"])
    return g


def _oracle(sc):
    o = OracleSolver(sc["cfg"], sc["sources"], sc["probes"], mask=sc["mask"], blend_xy=sc.get("blend_xy"),
                     field_xy=sc.get("field_xy"))
    if sc.get("rho0") is not None:
        o.set_density(sc["rho0"])
    return o


@pytest.mark.parametrize("name", ["lloyd_a", "doppler_a", "scattering_a", "hpc_a"])
def test_scheme_a_matches_oracle(name, gpu):
    sc = scenarios.family_a(name)
    g = _solver(sc)
    o = _oracle(sc)
    g.step(sc["steps"])
    o.step(sc["steps"])
    pg, po = g.get_probes(), o.get_probes()
    assert pg.shape == po.shape == (sc["steps"], len(sc["probes"]))
    assert np.max(np.abs(po)) > 0
    assert rel_l2(pg, po) <= PROBE_TOL, rel_l2(pg, po)
    nx, ny, nz = g.dims
    fo = (o.get_rho().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1] - 1.0)
    mask = o.get_mask().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1]
    fo[mask == 1] = 0.0
    fg = g.get_rho().astype(np.float64)
    assert np.max(np.abs(fg - fo)) <= FIELD_TOL * np.max(np.abs(fo))


@pytest.mark.parametrize("name", ["lloyd_a", "doppler_a", "scattering_a", "hpc_a"])
def test_scheme_a_matches_reference_fixture(name, gpu):
    path = os.path.join(GOLDEN, name + ".npz")
    gold = np.load(path)
    sc = scenarios.family_a(name, steps=int(gold["steps"]))
    g = _solver(sc)
    g.step(sc["steps"])
    nx, ny, nz = g.dims
    fg = g.get_rho().astype(np.float64).reshape(nz, ny, nx)
    ref = gold["rho_minus_1"]                       # reference's rho - 1 on interior cells, SOLID as 0
    assert np.max(np.abs(fg - ref)) <= FIELD_TOL * np.max(np.abs(ref))


def test_scheme_a_direct_calls_equal_batched_steps(gpu):
    sc = scenarios.family_a("doppler_a", steps=12)
    a = _solver(sc)
    a.step(sc["steps"])
    b = _solver(sc)
    for s in range(sc["steps"]):
        b.apply_source(s * b.dt)          # no-op for field sources: they act inside the step
        b.exchange_halos()                # no-op: each step writes the next step's halos
        b.step_collision_bgk()
        b.record_probes()
    assert np.array_equal(a.get_probes(), b.get_probes())
    assert np.array_equal(a.get_rho(), b.get_rho())


def test_scheme_a_solid_wall_direct_equals_batched(gpu):
    sc = scenarios.family_a("lloyd_a", steps=9)
    a = _solver(sc)
    a.step(sc["steps"])
    b = _solver(sc)
    for s in range(sc["steps"]):
        b.step_collision_bgk()
        b.record_probes()
    assert np.array_equal(a.get_probes(), b.get_probes())


def _scattering_3d(steps, **kw):
    """01's set-up with a pulse that varies along the periodic z axis, so
    the halo planes carry something the interior planes do not already hold."""
    sc = scenarios.scattering_a(steps=steps, z=(-0.4, 0.4), **kw)
    nx, ny, nz = 90, 60, 8
    zc = -0.4 + (np.arange(nz) + 0.5) * 0.1
    rho0 = sc["rho0"].reshape(nz, ny, nx) * (1.0 + 0.5 * np.cos(2.0 * np.pi * (zc - 0.13) / 0.8))[:, None, None]
    sc["rho0"] = rho0.ravel()
    return sc


def test_periodic_z_pulse_matches_oracle(gpu):
    sc = _scattering_3d(50)
    g, o = _solver(sc), _oracle(sc)
    g.step(sc["steps"])
    o.step(sc["steps"])
    assert rel_l2(g.get_probes(), o.get_probes()) <= PROBE_TOL
    nx, ny, nz = g.dims
    fo = o.get_rho().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1] - 1.0
    fo[o.get_mask().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1] == 1] = 0.0
    assert np.ptp(fo[:, 30, 70]) > 1e-4                  # the field still varies along z
    assert np.max(np.abs(g.get_rho().astype(np.float64) - fo)) <= FIELD_TOL * np.max(np.abs(fo))


def test_wall_faces_with_initial_pulse_match_oracle(gpu):
    """x faces SOLID (LBM_BC_WALL): the initial pulse reaches the high x wall,
    so the first steps bounce back from the slots lbm_set_density wrote into
    the x-face arrays; y faces SOLID too, periodic z."""
    sc = _scattering_3d(40)
    cfg = sc["cfg"]
    for f in range(4):
        cfg.face_bc[f] = abi.LBM_BC_WALL
    nx, ny, nz = 90, 60, 8
    mask = sc["mask"].reshape(nz + 2, ny + 2, nx + 2).copy()
    mask[:, :, 0] = mask[:, :, -1] = 1
    mask[:, 0, :] = mask[:, -1, :] = 1
    sc["mask"] = mask.ravel()
    g, o = _solver(sc), _oracle(sc)
    assert np.array_equal(g.get_mask(), o.get_mask())
    g.step(sc["steps"])
    o.step(sc["steps"])
    assert rel_l2(g.get_probes(), o.get_probes()) <= PROBE_TOL
    fo = o.get_rho().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1] - 1.0
    fo[o.get_mask().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1] == 1] = 0.0
    assert np.max(np.abs(fo[:, :, -1])) > 1e-5              # the wave is at the x wall
    assert np.max(np.abs(g.get_rho().astype(np.float64) - fo)) <= FIELD_TOL * np.max(np.abs(fo))


def test_copy_halos_with_initial_pulse_match_oracle(gpu):
    """Zero-gradient halos (03) and background flow with an initial density
    pulse that already covers the high x face: the first step pulls the
    halo copies of the pulse, not rest."""
    sc = scenarios.family_a("doppler_a", steps=30)
    n, dx = 40, 0.25
    c = (np.arange(n) + 0.5) * dx
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    sc["rho0"] = (1e-3 * np.exp(-((x - (n * dx - 0.6)) ** 2 + (y - 5.0) ** 2 + (z - 5.0) ** 2) / 2.0)).ravel()
    sc["sources"] = []
    g, o = _solver(sc), _oracle(sc)
    g.step(sc["steps"])
    o.step(sc["steps"])
    assert rel_l2(g.get_probes(), o.get_probes()) <= PROBE_TOL
    fo = o.get_rho().reshape(n + 2, n + 2, n + 2)[1:-1, 1:-1, 1:-1] - 1.0
    assert np.max(np.abs(fo[:, :, -1])) > 1e-5
    assert np.max(np.abs(g.get_rho().astype(np.float64) - fo)) <= FIELD_TOL * np.max(np.abs(fo))


def test_periodic_z_direct_calls_equal_batched_steps(gpu):
    sc = _scattering_3d(10)
    a = _solver(sc)
    a.step(sc["steps"])
    b = _solver(sc)
    for s in range(sc["steps"]):
        b.step_collision_bgk()
        b.record_probes()
    assert np.array_equal(a.get_probes(), b.get_probes())
    assert np.array_equal(a.get_rho(), b.get_rho())


def test_set_density_rules(gpu):
    sc = scenarios.scattering_a(steps=2)
    g = _solver(sc)
    with pytest.raises(LBMError) as e:
        g.set_density(sc["rho0"][:-1])
    assert e.value.status == abi.LBM_ERR_INVALID_ARGUMENT
    g.step(1)
    with pytest.raises(LBMError) as e:
        g.set_density(sc["rho0"])
    assert e.value.status == abi.LBM_ERR_STATE
    b = Solver(scenarios.family_a("doppler_a")["cfg"], [], None)
    b.set_density(np.zeros(b.dims[0] * b.dims[1] * b.dims[2]))    # any scheme-A set-up
    lat = Solver(scenarios.lattice_config(16, 16, 8, 0.52, use_geometry=0), [], None)
    with pytest.raises(LBMError) as e:
        lat.set_density(np.zeros(16 * 16 * 8))
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED


@pytest.mark.parametrize("name", ["lloyd_a", "doppler_a"])
def test_column_source_weights_with_other_source_forms(name, gpu):
    """Per-column source weights (a line source) with 02's destination source
    and 03's forcing (and its zero-gradient halos, which take their nearest
    column's weight), against the oracle."""
    sc = scenarios.family_a(name, steps=40)
    cfg = sc["cfg"]
    nx = int(round((cfg.x_max - cfg.x_min) / cfg.dx))
    ny = int(round((cfg.y_max - cfg.y_min) / cfg.dx))
    s0 = sc["sources"][0]
    xc = cfg.x_min + (np.arange(nx) + 0.5) * cfg.dx
    yc = cfg.y_min + (np.arange(ny) + 0.5) * cfg.dx
    d2 = (xc[None, :] - s0.sx) ** 2 + (yc[:, None] - s0.sy) ** 2
    sc["field_xy"] = np.where(d2 > 4.0, 0.0, np.exp(-d2 / 0.5)).ravel()
    g, o = _solver(sc), _oracle(sc)
    g.step(sc["steps"])
    o.step(sc["steps"])
    assert np.max(np.abs(o.get_probes())) > 0
    assert rel_l2(g.get_probes(), o.get_probes()) <= PROBE_TOL
    nx_, ny_, nz_ = g.dims
    fo = o.get_rho().reshape(nz_ + 2, ny_ + 2, nx_ + 2)[1:-1, 1:-1, 1:-1] - 1.0
    fo[o.get_mask().reshape(nz_ + 2, ny_ + 2, nx_ + 2)[1:-1, 1:-1, 1:-1] == 1] = 0.0
    assert np.max(np.abs(g.get_rho().astype(np.float64) - fo)) <= FIELD_TOL * np.max(np.abs(fo))


def test_pre_step_source_direct_calls_equal_batched_steps(gpu):
    sc = scenarios.family_a("hpc_a", steps=12)
    a = _solver(sc)
    a.step(sc["steps"])
    b = _solver(sc)
    for s in range(sc["steps"]):
        b.step_collision_bgk()
        b.record_probes()
    assert np.array_equal(a.get_probes(), b.get_probes())
    assert np.array_equal(a.get_rho(), b.get_rho())


def test_column_field_rules(gpu):
    sc = scenarios.family_a("hpc_a", steps=2)
    n = 52
    with pytest.raises(LBMError) as e:                      # count
        Solver(sc["cfg"], sc["sources"], None, mask=sc["mask"], blend_xy=np.zeros(n * n - 1))
    assert e.value.status == abi.LBM_ERR_INVALID_ARGUMENT
    lat = scenarios.lattice_config(16, 16, 8, 0.52, use_geometry=0)
    with pytest.raises(LBMError) as e:                      # scheme B
        Solver(lat, [], None, field_xy=np.zeros(16 * 16))
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
    c = sc["cfg"]
    c.sponge_blend = 0
    with pytest.raises(LBMError) as e:                      # blend strengths without the blend
        Solver(c, sc["sources"], None, mask=sc["mask"], blend_xy=sc["blend_xy"])
    assert e.value.status == abi.LBM_ERR_BAD_CONFIG
    c.sponge_blend = 1
    g = _solver(sc)
    a = np.ascontiguousarray(sc["blend_xy"], dtype=np.float64)
    assert g.lib.lbm_set_blend_xy(g.h, a.ctypes.data_as(abi.c_double_p), a.size) == abi.LBM_ERR_STATE   # after init
    src = abi.LbmSource()
    ctypes.pointer(src)[0] = sc["sources"][0]
    src.waveform = abi.LBM_WAVE_GAUSS                     # nonzero at t = 0
    src.t0, src.sigma_t = 0.0, 1.0
    with pytest.raises(LBMError) as e:
        Solver(c, [src], None, mask=sc["mask"], field_xy=sc["field_xy"], blend_xy=sc["blend_xy"])
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED


def test_uniform_flow_is_steady(gpu):
    sc = scenarios.family_a("doppler_a", steps=40)
    g = Solver(sc["cfg"], [], sc["probes"])     # no source: feq(1, flow) everywhere is a fixed point
    g.step(sc["steps"])
    assert np.max(np.abs(g.get_probes())) <= 1e-6
    assert np.max(np.abs(g.get_rho())) <= 1e-6


def test_scheme_a_rejects_unsupported_set_ups(gpu):
    sc = scenarios.family_a("doppler_a")
    cfg = sc["cfg"]
    for bad in (dict(storage=abi.LBM_STORE_F16, f16_scale=100.0), dict(face_bc=(abi.LBM_BC_NSCBC,) * 6),
                dict(face_bc=(abi.LBM_BC_COPY,) * 5 + (abi.LBM_BC_REST,)), dict(tau_sponge_max=0.505)):
        c = abi.reference_config(**{f[0]: getattr(cfg, f[0]) for f in abi.LbmConfig._fields_
                                    if f[0] not in ("face_bc", "flow")},
                                 face_bc=tuple(cfg.face_bc), flow=tuple(cfg.flow))
        for k, v in bad.items():
            if k == "face_bc":
                for f in range(6):
                    c.face_bc[f] = v[f]
            else:
                setattr(c, k, v)
        with pytest.raises(LBMError) as e:
            Solver(c, [], None)
        assert e.value.status == abi.LBM_ERR_BAD_CONFIG
    g = Solver(cfg, [], None)
    point = abi.reference_source(sx=5.0, sy=5.0, sz=5.0, ex=5.0, ey=5.0, ez=5.0)
    with pytest.raises(LBMError) as e:
        g.add_source(point)
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
    with pytest.raises(LBMError) as e:
        g.get_f()
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
