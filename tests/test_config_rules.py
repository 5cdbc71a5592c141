"""Configuration rules lbm_create enforces before any device work (runs
without a GPU): scheme A limits (periodic z, the destination blend sponge)
and z-slab bounds."""
import ctypes

import pytest

import nlos_lbm
import scenarios
from nlos_lbm import abi


def _create(cfg):
    lib = nlos_lbm.library()
    h = ctypes.c_void_p()
    st = lib.lbm_create(ctypes.byref(cfg), ctypes.byref(h))
    if h:
        lib.lbm_destroy(h)
    return st


def _cfg(**kw):
    return scenarios.lattice_config(32, 24, 16, 0.52, **kw)


@pytest.mark.parametrize("kw", [
    dict(scheme=abi.LBM_SCHEME_A, storage=abi.LBM_STORE_F16, f16_scale=10.0),   # scheme A is FP32
    dict(scheme=abi.LBM_SCHEME_A),                                               # NSCBC faces (the default)
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_COPY,) * 3 + (abi.LBM_BC_REST,) * 3),
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 6, tau_sponge_max=0.51),
    dict(face_bc=(abi.LBM_BC_COPY,) * 6),                                        # COPY needs scheme A
    dict(scheme=7),
    dict(dt=-1.0),
    dict(slab_k0=10, slab_nz=8),                                                 # past the 16 layers
    dict(slab_k0=-1, slab_nz=4),
    dict(slab_k0=0, slab_nz=8, scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 6),
    dict(face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2),          # periodic needs scheme A
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_PERIODIC,) * 2 + (abi.LBM_BC_REST,) * 4),   # z only
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 5 + (abi.LBM_BC_PERIODIC,)),      # both z faces
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 6, sponge_blend=1, tau_sponge_max=1.0),
    dict(face_bc=(abi.LBM_BC_REST,) * 6, sponge_blend=1),                        # blend needs scheme A
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 6, sponge_blend=2),
    dict(face_bc=(5,) * 6),
])
def test_rejected_configs(kw):
    assert _create(_cfg(**kw)) == abi.LBM_ERR_BAD_CONFIG


@pytest.mark.parametrize("kw", [
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 6, tau_sponge_max=1.0),
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_COPY,) * 6, flow=(0.0, 0.0, 0.1)),
    dict(slab_k0=8, slab_nz=8),
    dict(scheme=abi.LBM_SCHEME_A, face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2, sponge_blend=1),
])
def test_accepted_configs(kw):
    # without a GPU the device check comes after validation
    assert _create(_cfg(**kw)) in (abi.LBM_OK, abi.LBM_ERR_NO_DEVICE)
