"""Host geometry: the product voxeliser is bit-identical to the oracle (and
to the reference where its harness is built); STL output round-trips; the
synthetic city generator meets its stated properties."""
import numpy as np
import pytest

import nlos_lbm
import oracle
import scenarios
from nlos_lbm import abi


@pytest.mark.parametrize("seed,dims,sky", [(3, (160, 128, 48), 1e30), (11, (200, 150, 60), 25.0),
                                           (29, (96, 96, 40), 120.0)])
def test_voxelizer_matches_oracle(seed, dims, sky, tmp_path):
    nx, ny, nz = dims
    tris, _ = nlos_lbm.city_triangles(nx, ny, seed=seed, height=(10, 50), fp=(12, 40))
    cfg = abi.reference_config(x_min=0, x_max=nx, y_min=0, y_max=ny, z_min=0, z_max=nz, dx=1.0, sky_z=sky)
    m = nlos_lbm.voxelize(cfg, tris)
    stl = str(tmp_path / "c.stl")
    nlos_lbm.stl_write(stl, tris)
    o = oracle.OracleSolver(cfg, [], None, stl=stl)
    assert np.array_equal(m, o.get_mask())
    assert m.sum() > 0


def test_voxelizer_offsets_and_spacing_match_oracle():
    """Non-unit spacing, shifted origin and an STL offset (06:90-92, 06:464-476)."""
    tris = oracle.box_triangles([(3.0, 4.0, 0.0, 17.0, 11.0, 9.0), (20.5, 2.0, -1.0, 30.0, 18.0, 14.0)])
    off = (-1.25, 0.5, 0.0)
    cfg = abi.reference_config(x_min=-2.0, x_max=34.0, y_min=-1.0, y_max=23.0, z_min=0.0, z_max=18.0, dx=1.5)
    m = nlos_lbm.voxelize(cfg, tris, stl_offset=off)
    o = oracle.OracleSolver(cfg, [], None, triangles=tris, stl_offset=off)
    assert np.array_equal(m, o.get_mask())


def test_voxelizer_face_walls_and_no_geometry():
    cfg = scenarios.lattice_config(12, 10, 8, 0.6, face_bc=(abi.LBM_BC_WALL, abi.LBM_BC_NSCBC, abi.LBM_BC_REST,
                                                            abi.LBM_BC_WALL, abi.LBM_BC_NSCBC, abi.LBM_BC_WALL),
                                   use_geometry=0)
    m = nlos_lbm.voxelize(cfg, None).reshape(10, 12, 14)
    o = oracle.OracleSolver(cfg, [], None)
    assert np.array_equal(m.ravel(), o.get_mask())
    assert m[5, 5, 0] == 1 and m[5, 5, 13] == 0 and m[5, 11, 5] == 1 and m[9, 5, 5] == 1
    assert m[1:-1, 1:-1, 1:-1].sum() == 0


@pytest.mark.skipif(not oracle.ref_available("06"), reason="reference harness not built here")
def test_voxelizer_matches_live_reference(tmp_path):
    nx, ny, nz = 128, 96, 40
    tris, _ = nlos_lbm.city_triangles(nx, ny, seed=42, height=(5, 35), fp=(10, 30), street=6)
    stl = str(tmp_path / "c.stl")
    nlos_lbm.stl_write(stl, tris)
    cfg = abi.reference_config(x_min=0, x_max=nx, y_min=0, y_max=ny, z_min=0, z_max=nz, dx=1.0)
    ref = oracle.RefSolver("06", (0, nx), (0, ny), (0, nz), 1.0, 0.55, (1, 1, 1, 1, 1, 1, 0, 0, 0), stl=stl)
    assert np.array_equal(nlos_lbm.voxelize(cfg, tris), ref.get_mask())


def test_stl_round_trip_through_reference_loader_layout(tmp_path):
    tris, _ = nlos_lbm.city_triangles(64, 64, seed=1, fp=(10, 20), height=(5, 9), street=4)
    p = str(tmp_path / "x.stl")
    nlos_lbm.stl_write(p, tris)
    raw = open(p, "rb").read()
    n = int.from_bytes(raw[80:84], "little")
    assert n == len(tris) and len(raw) == 84 + 50 * n
    rec = np.frombuffer(raw[84:], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    np.testing.assert_array_equal(rec["v"], tris)
    nrm = rec["n"]
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, rtol=1e-6)


def test_missing_stl_gives_empty_geometry_like_reference(tmp_path):
    """GeometryEngine::load fails -> empty geometry, run continues (06:397-410)."""
    cfg = scenarios.lattice_config(10, 10, 10, 0.6)
    o = oracle.OracleSolver(cfg, [], None, stl=str(tmp_path / "nope.stl"))
    assert o.stl_status == abi.LBM_WARN_STL_NOT_LOADED
    assert np.array_equal(o.get_mask(), nlos_lbm.voxelize(cfg, None))


def test_city_generator_properties():
    p = dict(fp=(20, 60), height=(10, 80), coverage=0.40, street=8)
    a, cov = nlos_lbm.city_triangles(1024, 1024, seed=2024, **p)
    b, cov2 = nlos_lbm.city_triangles(1024, 1024, seed=2024, **p)
    c, _ = nlos_lbm.city_triangles(1024, 1024, seed=2025, **p)
    assert np.array_equal(a, b) and cov == cov2          # seeded, deterministic
    assert not np.array_equal(a[: min(len(a), len(c))], c[: min(len(a), len(c))])
    assert 0.40 <= cov < 0.5
    assert len(a) % 12 == 0
    boxes = a.reshape(-1, 12, 3, 3)
    lo = boxes.min(axis=(1, 2))
    hi = boxes.max(axis=(1, 2))
    w = hi - lo
    assert np.all((w[:, 0] >= 20) & (w[:, 0] <= 60) & (w[:, 1] >= 20) & (w[:, 1] <= 60))
    assert np.all((w[:, 2] >= 10) & (w[:, 2] <= 80)) and np.all(lo[:, 2] == 0)
    assert np.all(lo == np.round(lo)) and np.all(hi == np.round(hi))   # vertices on the lattice
    # streets: any two footprints are at least 8 cells apart along x or y
    n = len(lo)
    for i in range(n):
        gx = np.maximum(lo[:, 0] - hi[i, 0], lo[i, 0] - hi[:, 0])
        gy = np.maximum(lo[:, 1] - hi[i, 1], lo[i, 1] - hi[:, 1])
        gap = np.maximum(gx, gy)
        gap[i] = np.inf
        assert gap.min() >= 8


@pytest.mark.skipif(not oracle.ref_available("06"), reason="reference harness not built here")
@pytest.mark.parametrize("keep,extra", [(30, 0), (30, 17)])
def test_truncated_stl_oracle_matches_live_reference(keep, extra, tmp_path):
    """GeometryEngine::load on a file shorter than its header's count (06:74-85):
    the missing bytes stay zero.  The oracle reads it the same way, which the
    GPU tests then hold the library's mask to."""
    nx, ny, nz = 96, 80, 40
    tris, _ = nlos_lbm.city_triangles(nx, ny, seed=7, height=(5, 30), fp=(10, 24), street=6)
    path = str(tmp_path / "t.stl")
    nlos_lbm.stl_write(path, tris)
    raw = open(path, "rb").read()
    open(path, "wb").write(raw[:84 + 50 * keep + extra])
    cfg = abi.reference_config(x_min=0, x_max=nx, y_min=0, y_max=ny, z_min=0, z_max=nz, dx=1.0)
    ref = oracle.RefSolver("06", (0, nx), (0, ny), (0, nz), 1.0, 0.55, (1, 1, 1, 1, 1, 1, 0, 0, 0), stl=path)
    o = oracle.OracleSolver(cfg, [], None, stl=path)
    assert np.array_equal(o.get_mask(), ref.get_mask())
    assert o.get_mask().sum() > 0
