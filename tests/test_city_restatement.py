"""The pure-Python city generator of oracle/city.py (used by the reference arm
of bench.py, which must not load the product library) produces the product
generator's triangles bit for bit, and a window cropped from a city
voxelises to the same mask as that window of the whole city."""
import numpy as np
import pytest

import nlos_lbm
from nlos_lbm import abi
from oracle import city


@pytest.mark.parametrize("nx,ny,seed,kw", [
    (2048, 2048, 2024, dict(fp=(20, 60), height=(10, 80), coverage=0.40, street=8, margin=40)),   # the C4 city
    (512, 384, 7, dict(fp=(12, 40), height=(5, 30), coverage=0.5, street=6, margin=0)),
    (96, 80, 3, dict(fp=(10, 24), height=(5, 30), coverage=0.3, street=6, margin=4)),
])
def test_city_restatement_matches_product_generator(nx, ny, seed, kw):
    got, cov = city.city_triangles(nx, ny, seed, **kw)
    ref, cov_ref = nlos_lbm.city_triangles(nx, ny, seed=seed, **kw)
    assert got.dtype == np.float32 and got.shape == ref.shape
    assert np.array_equal(got, ref)
    assert cov == cov_ref


def test_cropped_window_voxelises_like_the_whole_city():
    nx, ny, nz = 512, 512, 96
    boxes, _ = city.city_boxes(nx, ny, 2024, fp=(20, 60), height=(10, 80), coverage=0.40, street=8, margin=40)
    whole = np.concatenate([city.box_triangles(*b) for b in boxes])
    cfg = abi.reference_config(x_min=0, x_max=nx, y_min=0, y_max=ny, z_min=0, z_max=nz, dx=1.0)
    m = nlos_lbm.voxelize(cfg, whole).reshape(nz + 2, ny + 2, nx + 2)
    x0, y0, w = 128, 160, 256
    part = city.crop_boxes(boxes, x0, y0, x0 + w, y0 + w)
    tris = np.concatenate([city.box_triangles(*b) for b in part])
    cfg_w = abi.reference_config(x_min=0, x_max=w, y_min=0, y_max=w, z_min=0, z_max=nz, dx=1.0)
    mw = nlos_lbm.voxelize(cfg_w, tris).reshape(nz + 2, w + 2, w + 2)
    # interior columns of the window (the halo columns border different neighbours)
    assert np.array_equal(mw[:, 1:-1, 1:-1], m[:, y0 + 1:y0 + w + 1, x0 + 1:x0 + w + 1])
    assert mw[1:-1, 1:-1, 1:-1].sum() > 0


def test_python_stl_writer_matches_product_writer(tmp_path):
    tris, _ = city.city_triangles(128, 128, 5, fp=(10, 30), height=(5, 20), street=6)
    a, b = str(tmp_path / "a.stl"), str(tmp_path / "b.stl")
    city.stl_write(a, tris)
    nlos_lbm.stl_write(b, tris)
    ra, rb = open(a, "rb").read(), open(b, "rb").read()
    assert ra[80:] == rb[80:]   # everything after the free-text header
