"""lbm_get_rho_noalloc: the field-output entry point that allocates nothing.

It exists for callers that cannot allocate device memory when they read a
field (an application whose own memory pool owns the GPU, or a frame loop
that must not stall on cudaMalloc/cudaFree synchronisation).  Its output
must equal that of the allocating lbm_get_rho, on consecutive calls, and
across handles of different sizes that share its static device array.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import nlos_lbm
import scenarios
from nlos_lbm import abi

pytestmark = pytest.mark.gpu

def rho_alloc(s):
    return s.get_rho().ravel()


def rho_noalloc(s):
    nx, ny, nz = s.dims
    out = np.empty(nx * ny * nz, dtype=np.float32)
    st = s.lib.lbm_get_rho_noalloc(s.h, out.ctypes.data_as(abi.c_float_p), out.size)
    assert st == abi.LBM_OK, (st, s.lib.lbm_last_error(s.h))
    return out


def same(a, b):
    """Both entry points run the same field kernel on the same state: the
    results must be equal bit for bit, and not trivially zero."""
    assert a.shape == b.shape
    assert np.array_equal(a, b)
    assert np.max(np.abs(b)) > 0


def test_noalloc_field_matches_allocating_call_twice_in_a_row(gpu):
    big = scenarios.scenario("city_small")          # 96 x 80 x 40 cells
    small = scenarios.scenario("lloyd_small")       # 64 x 32 x 32 cells
    a = nlos_lbm.Solver(big["cfg"], big["sources"], big["probes"], triangles=big["triangles"])
    b = nlos_lbm.Solver(small["cfg"], small["sources"], small["probes"], triangles=small["triangles"])
    a.step(60)
    b.step(45)
    # two calls in a row on one handle
    first, second = rho_noalloc(a), rho_noalloc(a)
    ref_a = rho_alloc(a)
    same(first, ref_a)
    same(second, ref_a)
    # a smaller grid after a larger one: the shared array's leftovers must not leak
    same(rho_noalloc(b), rho_alloc(b))
    # state moves on: the next call returns the new field
    a.step(7)
    same(rho_noalloc(a), rho_alloc(a))
    # FP16 storage goes through the same path
    h16 = scenarios.scenario("scatter_small", storage=abi.LBM_STORE_F16, f16_scale=1e3)
    c = nlos_lbm.Solver(h16["cfg"], h16["sources"], h16["probes"], triangles=h16["triangles"])
    c.step(40)
    same(rho_noalloc(c), rho_alloc(c))


def test_noalloc_field_of_scheme_a_with_initial_pulse(gpu):
    """01's set-up (scheme A, initial density pulse, periodic z): before the
    first step both entry points return the pulse at FLUID cells (01:197),
    after steps the scheme-A field kernel's output, through the static array."""
    sc = scenarios.scattering_a(steps=20)
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], mask=sc.get("mask"))
    g.set_density(sc["rho0"])
    before = rho_noalloc(g)
    same(before, rho_alloc(g))
    nx, ny, nz = g.dims
    mask = g.get_mask().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1].ravel()   # interior, i fastest
    pulse = np.asarray(sc["rho0"], dtype=np.float64).ravel().astype(np.float32)
    assert np.array_equal(before, np.where(mask == 1, np.float32(0), pulse))
    g.step(5)
    first, second = rho_noalloc(g), rho_noalloc(g)
    same(first, rho_alloc(g))
    same(second, first)
    assert not np.array_equal(first, before)


def test_noalloc_rejects_grids_beyond_its_array(gpu):
    nx, ny, nz = 256, 256, 129                      # 8,454,144 cells > 2^23
    assert nx * ny * nz > abi.LBM_NOALLOC_MAX_CELLS
    cfg = scenarios.lattice_config(nx, ny, nz, 0.6, storage=abi.LBM_STORE_F16, f16_scale=1e3)
    s = nlos_lbm.Solver(cfg, [], None)
    s.step(1)
    out = np.empty(nx * ny * nz, dtype=np.float32)
    st = s.lib.lbm_get_rho_noalloc(s.h, out.ctypes.data_as(abi.c_float_p), out.size)
    assert st == abi.LBM_ERR_UNSUPPORTED
    assert b"at most 8388608" in s.lib.lbm_last_error(s.h)
