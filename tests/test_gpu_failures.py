"""Failure paths of the library, made on the host: a non-finite state, a grid
larger than the device and a truncated STL file.  The reference fails
silently in all three (06:397-410 loads what it can, 06:432-435 only warns,
nothing checks the field); the library reports each with a status.  Nothing
here faults the GPU: a NaN is plain arithmetic, and the oversized grid is
refused before any allocation."""
import math

import numpy as np
import pytest

import nlos_lbm
import oracle
import scenarios
from nlos_lbm import LBMError, abi

pytestmark = pytest.mark.gpu


def poison_probe_cell(g, sc, probe=0, half=2):
    """NaN in every population of the (2 half + 1)^3 cells around a probe."""
    cfg = sc["cfg"]
    nxt, nyt, nzt = g.dims_halo
    x, y, z = np.asarray(sc["probes"], dtype=np.float64).reshape(-1, 3)[probe]
    ijk = [int(math.floor((v - lo) / cfg.dx)) + 1 for v, lo in ((x, cfg.x_min), (y, cfg.y_min), (z, cfg.z_min))]
    f = g.get_f().reshape(nzt, nyt, nxt, 19)
    i, j, k = ijk
    f[max(k - half, 1):k + half + 1, max(j - half, 1):j + half + 1, max(i - half, 1):i + half + 1, :] = np.nan
    g.set_f(f.ravel())


@pytest.mark.parametrize("storage", [abi.LBM_STORE_F32, abi.LBM_STORE_F16])
def test_non_finite_state_is_reported_by_the_step_call(storage, gpu):
    sc = scenarios.scenario("lloyd_small", storage=storage, f16_scale=1e3)
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(4)
    poison_probe_cell(g, sc)
    # the call in which the value appears returns LBM_ERR_NAN, steps taken
    with pytest.raises(LBMError) as e:
        g.step(6)
    assert e.value.status == abi.LBM_ERR_NAN
    assert g.lib.lbm_get_step(g.h) == 10
    assert b"non-finite" in g.lib.lbm_last_error(g.h)
    # the state stays flagged: the next call reports it too
    with pytest.raises(LBMError) as e:
        g.step(1)
    assert e.value.status == abi.LBM_ERR_NAN


def test_finite_run_is_not_flagged(gpu):
    sc = scenarios.scenario("lloyd_small")
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(50)
    assert np.all(np.isfinite(g.get_probes()))


def test_non_finite_state_in_standalone_calls_is_reported_at_the_next_step(gpu):
    """The reference's own call sequence (apply_source, exchange_halos,
    step_collision_bgk, record_probes) is not synchronised per call; the
    flag is read at the next lbm_step or lbm_get_probes."""
    sc = scenarios.scenario("lloyd_small")
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(2)
    poison_probe_cell(g, sc)
    for s in range(2, 5):
        g.apply_source(s * g.dt)
        g.exchange_halos()
        g.step_collision_bgk()
        g.record_probes()
    with pytest.raises(LBMError) as e:
        g.get_probes()
    assert e.value.status == abi.LBM_ERR_NAN


def test_grid_beyond_device_memory_is_refused_without_a_leak(gpu):
    import torch

    before = torch.cuda.mem_get_info(0)[0]
    # 2048 x 2048 x 320 FP32: two population buffers of 204 GB
    cfg = scenarios.lattice_config(2048, 2048, 320, 0.6)
    with pytest.raises(LBMError) as e:
        nlos_lbm.Solver(cfg, [], None)
    assert e.value.status == abi.LBM_ERR_OUT_OF_MEMORY
    assert "GB of device memory" in str(e.value)
    after = torch.cuda.mem_get_info(0)[0]
    assert abs(after - before) < 64 << 20
    # the library is still usable
    sc = scenarios.scenario("lloyd_small")
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(10)
    assert np.max(np.abs(g.get_probes())) > 0


def truncated_stl(path, tris, keep_records, extra_bytes=0, count=None):
    """Binary STL whose header counts `count` triangles (all of them by
    default) but which holds only `keep_records` records plus a few bytes."""
    nlos_lbm.stl_write(path, tris)
    raw = bytearray(open(path, "rb").read())
    n = len(tris) if count is None else count
    raw[80:84] = int(n).to_bytes(4, "little")
    open(path, "wb").write(bytes(raw[:84 + 50 * keep_records + extra_bytes]))


@pytest.mark.parametrize("keep,extra", [(30, 0), (30, 17), (0, 0)])
def test_truncated_stl_warns_and_matches_the_oracle_mask(keep, extra, tmp_path, gpu):
    """The library reads what the file holds; the records past its end are
    zero triangles as in the reference (a degenerate triangle at the offset
    point, which only widens the bin grid's bounding box), so the mask is
    the oracle's, which reads the header's count of records one by one."""
    nx, ny, nz = 96, 80, 40
    tris, _ = nlos_lbm.city_triangles(nx, ny, seed=7, height=(5, 30), fp=(10, 24), street=6)
    path = str(tmp_path / "t.stl")
    truncated_stl(path, tris, keep, extra)
    off = (3.0, 4.0, 0.0)
    cfg = scenarios.lattice_config(nx, ny, nz, 0.6)
    g = nlos_lbm.Solver(cfg, [], None, stl=path, stl_offset=off)
    assert abi.LBM_WARN_STL_TRUNCATED in g.warnings
    assert g.init_status == abi.LBM_WARN_STL_TRUNCATED
    o = oracle.OracleSolver(cfg, [], None, stl=path, stl_offset=off)
    assert np.array_equal(g.get_mask(), o.get_mask())


def test_stl_with_a_corrupt_count_allocates_only_what_the_file_holds(tmp_path, gpu):
    """A header that counts 2^32 - 1 triangles over a 40-record file: the
    reference would try to allocate them all; the library keeps 41."""
    tris, _ = nlos_lbm.city_triangles(64, 64, seed=5, height=(5, 20), fp=(10, 20), street=6)
    path = str(tmp_path / "c.stl")
    truncated_stl(path, tris, 40, 0, count=0xFFFFFFFF)
    cfg = scenarios.lattice_config(64, 64, 32, 0.6)
    g = nlos_lbm.Solver(cfg, [], None, stl=path)
    assert g.init_status == abi.LBM_WARN_STL_TRUNCATED
    # the same 40 records with a count of 41 give the same mask (one zero record)
    path2 = str(tmp_path / "c41.stl")
    truncated_stl(path2, tris, 40, 0, count=41)
    o = oracle.OracleSolver(cfg, [], None, stl=path2)
    assert np.array_equal(g.get_mask(), o.get_mask())
