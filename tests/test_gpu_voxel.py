"""The GPU heightmap voxeliser (voxel.cu, used by lbm_init) against the host
voxeliser (lbm_voxelize, HeightField::ground_height, itself bit-identical to
the reference's GeometryEngine in tests/test_geometry.py): the masks must be
bit-identical, on the synthetic city and on a dense sloped terrain mesh
whose rays hit triangles at arbitrary barycentric positions."""
import numpy as np
import pytest

import nlos_lbm
import scenarios
from nlos_lbm import Solver, abi

pytestmark = pytest.mark.gpu


def terrain_triangles(n, extent, seed, z0=2.0, amp=6.0):
    """A triangulated height field: n x n vertices over [0, extent]^2 with a
    seeded smooth random surface, two triangles per quad."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, extent, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    Z = z0 + amp * (0.5 + 0.25 * np.sin(X / 7.3 + rng.uniform(0, 6)) * np.cos(Y / 5.1 + rng.uniform(0, 6))
                    + 0.25 * rng.random((n, n)))
    v = np.stack([X, Y, Z], -1)
    a, b, c, d = v[:-1, :-1], v[1:, :-1], v[1:, 1:], v[:-1, 1:]
    t1 = np.concatenate([a, b, c], -1).reshape(-1, 9)
    t2 = np.concatenate([a, c, d], -1).reshape(-1, 9)
    return np.concatenate([t1, t2]).astype(np.float32)


def _masks(cfg, tris, offset=(0.0, 0.0, 0.0)):
    g = Solver(cfg, [], None, triangles=tris, stl_offset=offset)
    gm = g.get_mask()
    g.close()
    hm = nlos_lbm.voxelize(cfg, tris, stl_offset=offset)
    return gm, hm


def test_city_mask_matches_host(gpu):
    tris, _ = nlos_lbm.city_triangles(400, 300, seed=3, fp=(12, 30), height=(5, 40), street=6, margin=4)
    cfg = scenarios.lattice_config(400, 300, 48, 0.51)
    gm, hm = _masks(cfg, tris)
    assert gm.sum() > 0
    assert np.array_equal(gm, hm)


@pytest.mark.parametrize("seed", [0, 1])
def test_dense_terrain_mask_matches_host(seed, gpu):
    tris = terrain_triangles(181, 95.0, seed)          # 64,800 triangles, vertices off the cell centres
    cfg = scenarios.lattice_config(96, 96, 16, 0.51, dx=1.0, x_max=96.0, y_max=96.0, z_max=16.0)
    gm, hm = _masks(cfg, tris, offset=(0.37, -0.21, 0.0))
    assert 0 < gm.sum() < gm.size
    assert np.array_equal(gm, hm)


def test_no_geometry_and_empty_mesh(gpu):
    cfg = scenarios.lattice_config(40, 30, 20, 0.51)
    gm, hm = _masks(cfg, np.zeros((0, 9), np.float32))
    assert np.array_equal(gm, hm)
    cfg.use_geometry = 0
    gm, hm = _masks(cfg, terrain_triangles(21, 39.0, 2))
    assert np.array_equal(gm, hm)
