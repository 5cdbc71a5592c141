"""The C-ABI library loads on a host without a GPU and exports what
include/nlos_lbm.h declares; host-only entry points behave as documented."""
import ctypes
import os
import re

import numpy as np
import pytest

import nlos_lbm
from nlos_lbm import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "nlos_lbm.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void|double|long|const char\*)\s+(lbm_[a-z0-9_]+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(abi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_checked_library_exports_the_same_symbols():
    """liblbm_b200_check.so (-DLBM_CHECK) is a drop-in twin of the product library."""
    lib = ctypes.CDLL(os.path.join(abi.PACKAGE_DIR, "liblbm_b200_check.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    bound = set()

    class Rec:
        def __getattr__(self, n):
            bound.add(n)
            return type("F", (), {"restype": None, "argtypes": None})()

    abi.bind_product(Rec())
    assert set(declared_functions()) <= bound


def test_config_defaults_are_the_reference_values():
    lib = nlos_lbm.library()
    c = abi.LbmConfig()
    lib.lbm_config_default(ctypes.byref(c))
    r = abi.reference_config()
    for name, _ in abi.LbmConfig._fields_:
        a, b = getattr(c, name), getattr(r, name)
        if name in ("face_bc", "flow"):
            assert list(a) == list(b), name
        else:
            assert a == b, name
    assert (c.x_max, c.y_max, c.z_max, c.dx, c.tau) == (1650.0, 1150.0, 250.0, 2.0, 0.55)   # 06:250-268
    assert (c.sponge_width, c.sponge_strength, c.sky_z) == (20.0, 0.35, 120.0)             # 06:455-458
    assert c.face_bc[abi.FACE_ZLO] == abi.LBM_BC_WALL                                       # 06:520-531
    s = abi.LbmSource()
    lib.lbm_source_default(ctypes.byref(s))
    assert (s.t0, s.sigma_t, s.radius, s.sigma_cells, s.gain) == (0.05, 0.005, 2, 1.25, 1.0)   # 06:579-588


def test_status_strings():
    lib = nlos_lbm.library()
    for code in (0, 1, 2, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10):
        assert lib.lbm_status_string(code) != b"unknown status"
    assert lib.lbm_status_string(12345) == b"unknown status"


def test_create_rejects_bad_config_before_touching_a_device():
    lib = nlos_lbm.library()
    h = ctypes.c_void_p()
    for kw in (dict(tau=0.5), dict(dx=0.0), dict(x_max=-1.0), dict(storage=7), dict(storage=1, f16_scale=0.0)):
        c = abi.reference_config(**kw)
        assert lib.lbm_create(ctypes.byref(c), ctypes.byref(h)) == abi.LBM_ERR_BAD_CONFIG
    assert lib.lbm_create(None, ctypes.byref(h)) == abi.LBM_ERR_INVALID_ARGUMENT


def test_create_without_gpu_reports_no_device():
    from conftest import _has_gpu

    if _has_gpu():
        pytest.skip("a GPU is present")
    lib = nlos_lbm.library()
    h = ctypes.c_void_p()
    c = abi.reference_config()
    assert lib.lbm_create(ctypes.byref(c), ctypes.byref(h)) == abi.LBM_ERR_NO_DEVICE


def test_solver_raises_loudly_without_device():
    from conftest import _has_gpu

    if _has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(nlos_lbm.LBMError):
        nlos_lbm.Solver(abi.reference_config())
