"""ctypes mirror of include/nlos_lbm.h (structs, enums, prototypes).

This module only describes the C-ABI; it never touches a GPU.  The
high-level solver in ``nlos_lbm.solver`` and the oracle bindings both use it.
"""
import ctypes
import os

c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_long_p = ctypes.POINTER(ctypes.c_long)

# lbm_status
LBM_OK = 0
LBM_WARN_STL_NOT_LOADED = 1
LBM_WARN_PROBE_IN_SOLID = 2
LBM_WARN_STL_TRUNCATED = 3
LBM_ERR_INVALID_ARGUMENT = -1
LBM_ERR_BAD_CONFIG = -2
LBM_ERR_OUT_OF_MEMORY = -3
LBM_ERR_CUDA = -4
LBM_ERR_NAN = -5
LBM_ERR_STATE = -6
LBM_ERR_CAPACITY = -7
LBM_ERR_NO_DEVICE = -8
LBM_ERR_IO = -9
LBM_ERR_UNSUPPORTED = -10
LBM_NOALLOC_MAX_CELLS = 8388608

LBM_BC_NSCBC, LBM_BC_REST, LBM_BC_WALL, LBM_BC_COPY, LBM_BC_PERIODIC = 0, 1, 2, 3, 4
LBM_SCHEME_B, LBM_SCHEME_A = 0, 1
LBM_FIELD_DST, LBM_FIELD_FORCE, LBM_FIELD_PRE = 0, 1, 2
FACE_XLO, FACE_XHI, FACE_YLO, FACE_YHI, FACE_ZLO, FACE_ZHI = range(6)
LBM_STORE_F32, LBM_STORE_F16 = 0, 1
LBM_WAVE_GAUSS, LBM_WAVE_SINE, LBM_WAVE_RICKER, LBM_WAVE_TABLE = 0, 1, 2, 3
LBM_INJECT_GAUSS, LBM_INJECT_TRILINEAR, LBM_INJECT_FIELD = 0, 1, 2

# Family-B lattice (06:21-31)
Q = 19
EX = (0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 0, 0, 0, 0)
EY = (0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1)
EZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1)
W = (1.0 / 3.0,) + (1.0 / 18.0,) * 6 + (1.0 / 36.0,) * 12
CS = 0.57735026918962576451


class LbmConfig(ctypes.Structure):
    _fields_ = [
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
        ("dx", ctypes.c_double),
        ("c_phys", ctypes.c_double),
        ("tau", ctypes.c_double),
        ("use_geometry", ctypes.c_int),
        ("face_bc", ctypes.c_int * 6),
        ("sponge_faces", ctypes.c_uint),
        ("sponge_width", ctypes.c_double),
        ("sponge_strength", ctypes.c_double),
        ("sky_z", ctypes.c_double),
        ("storage", ctypes.c_int),
        ("f16_scale", ctypes.c_double),
        ("device", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("scheme", ctypes.c_int),
        ("tau_sponge_max", ctypes.c_double),
        ("flow", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("slab_k0", ctypes.c_int),
        ("slab_nz", ctypes.c_int),
        ("sponge_blend", ctypes.c_int),
    ]


class LbmSource(ctypes.Structure):
    _fields_ = [
        ("sx", ctypes.c_double), ("sy", ctypes.c_double), ("sz", ctypes.c_double),
        ("ex", ctypes.c_double), ("ey", ctypes.c_double), ("ez", ctypes.c_double),
        ("speed", ctypes.c_double),
        ("amp", ctypes.c_double),
        ("freq", ctypes.c_double),
        ("waveform", ctypes.c_int),
        ("t0", ctypes.c_double), ("sigma_t", ctypes.c_double),
        ("injection", ctypes.c_int),
        ("gain", ctypes.c_double),
        ("sigma_cells", ctypes.c_double),
        ("radius", ctypes.c_int),
        ("table", c_double_p),
        ("table_len", ctypes.c_int),
        ("field_mode", ctypes.c_int),
    ]


class LbmCityParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("fp_min", ctypes.c_int), ("fp_max", ctypes.c_int),
        ("h_min", ctypes.c_int), ("h_max", ctypes.c_int),
        ("coverage", ctypes.c_double),
        ("street", ctypes.c_int),
        ("margin", ctypes.c_int),
    ]


def reference_config(**kw):
    """lbm_config with the reference's defaults (06:250-268, 06:455-458):
    NSCBC on x-, x+, y-, y+, z+, ground wall at z-, sponge on the open faces."""
    c = LbmConfig()
    c.x_min, c.x_max = 0.0, 1650.0
    c.y_min, c.y_max = 0.0, 1150.0
    c.z_min, c.z_max = 0.0, 250.0
    c.dx = 2.0
    c.c_phys = 340.0
    c.tau = 0.55
    c.use_geometry = 1
    for f in range(6):
        c.face_bc[f] = LBM_BC_NSCBC
    c.face_bc[FACE_ZLO] = LBM_BC_WALL
    c.sponge_faces = (1 << FACE_XLO) | (1 << FACE_XHI) | (1 << FACE_YLO) | (1 << FACE_YHI) | (1 << FACE_ZHI)
    c.sponge_width = 20.0
    c.sponge_strength = 0.35
    c.sky_z = 120.0
    c.storage = LBM_STORE_F32
    c.f16_scale = 1.0
    c.device = 0
    c.use_graphs = 1
    c.verbose = 0
    c.scheme = LBM_SCHEME_B
    c.tau_sponge_max = 0.0
    c.dt = 0.0
    for k, v in kw.items():
        if k == "flow":
            for a in range(3):
                c.flow[a] = v[a]
            continue
        if k == "face_bc":
            for f in range(6):
                c.face_bc[f] = v[f]
        else:
            setattr(c, k, v)
    return c


def reference_source(**kw):
    """lbm_source with the reference's defaults (06:579-588)."""
    s = LbmSource()
    s.waveform = LBM_WAVE_GAUSS
    s.t0, s.sigma_t = 0.05, 0.005
    s.injection = LBM_INJECT_GAUSS
    s.gain = 1.0
    s.sigma_cells = 1.25
    s.radius = 2
    s.table = None
    s.table_len = 0
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def bind_product(lib):
    """Declare the prototypes of include/nlos_lbm.h on a loaded CDLL."""
    P = ctypes.c_void_p
    sig = {
        "lbm_config_default": (None, [ctypes.POINTER(LbmConfig)]),
        "lbm_source_default": (None, [ctypes.POINTER(LbmSource)]),
        "lbm_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "lbm_version": (ctypes.c_char_p, []),
        "lbm_create": (ctypes.c_int, [ctypes.POINTER(LbmConfig), ctypes.POINTER(P)]),
        "lbm_destroy": (ctypes.c_int, [P]),
        "lbm_last_error": (ctypes.c_char_p, [P]),
        "lbm_set_geometry_stl": (ctypes.c_int, [P, ctypes.c_char_p] + [ctypes.c_double] * 4),
        "lbm_set_geometry_triangles": (ctypes.c_int, [P, c_float_p, ctypes.c_int] + [ctypes.c_double] * 4),
        "lbm_set_mask": (ctypes.c_int, [P, c_uint8_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "lbm_add_source": (ctypes.c_int, [P, ctypes.POINTER(LbmSource)]),
        "lbm_clear_sources": (ctypes.c_int, [P]),
        "lbm_set_probes": (ctypes.c_int, [P, c_double_p, ctypes.c_int]),
        "lbm_probe_info": (ctypes.c_int, [P, c_int_p, c_int_p]),
        "lbm_init": (ctypes.c_int, [P]),
        "lbm_apply_source": (ctypes.c_int, [P, ctypes.c_double]),
        "lbm_exchange_halos": (ctypes.c_int, [P]),
        "lbm_step_collision_bgk": (ctypes.c_int, [P]),
        "lbm_record_probes": (ctypes.c_int, [P]),
        "lbm_step": (ctypes.c_int, [P, ctypes.c_int]),
        "lbm_run": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_int]),
        "lbm_synchronize": (ctypes.c_int, [P]),
        "lbm_get_dims": (ctypes.c_int, [P, c_int_p, c_int_p]),
        "lbm_get_dt": (ctypes.c_double, [P]),
        "lbm_get_step": (ctypes.c_long, [P]),
        "lbm_get_probes": (ctypes.c_int, [P, c_double_p, ctypes.c_long, c_long_p]),
        "lbm_get_probe_energy": (ctypes.c_int, [P, c_double_p]),
        "lbm_get_rho": (ctypes.c_int, [P, c_float_p, ctypes.c_long]),
        "lbm_get_rho_noalloc": (ctypes.c_int, [P, c_float_p, ctypes.c_long]),
        "lbm_get_f": (ctypes.c_int, [P, c_double_p, ctypes.c_long]),
        "lbm_set_f": (ctypes.c_int, [P, c_double_p, ctypes.c_long]),
        "lbm_set_density": (ctypes.c_int, [P, c_double_p, ctypes.c_long]),
        "lbm_set_blend_xy": (ctypes.c_int, [P, c_double_p, ctypes.c_long]),
        "lbm_set_field_weights_xy": (ctypes.c_int, [P, c_double_p, ctypes.c_long]),
        "lbm_get_mask": (ctypes.c_int, [P, c_uint8_p, ctypes.c_long]),
        "lbm_set_kernel_timing": (ctypes.c_int, [P, ctypes.c_int]),
        "lbm_get_kernel_time": (ctypes.c_int, [P, c_double_p, c_long_p]),
        "lbm_get_launch_count": (ctypes.c_long, [P]),
        "lbm_bytes_per_cell": (ctypes.c_int, [P]),
        "lbm_get_stream": (ctypes.c_void_p, [P]),
        "lbm_get_transfer_bytes": (ctypes.c_int, [P, c_long_p, c_long_p]),
        "lbm_check_status": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "lbm_check_selftest": (ctypes.c_int, [P]),
        "lbm_adjoint_grad": (ctypes.c_int, [P, ctypes.c_int, c_double_p, ctypes.c_int, ctypes.c_int, c_double_p,
                                            c_double_p, c_double_p, c_double_p]),
        "lbm_adjoint_plan": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p, c_int_p,
                                            ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "lbm_adjoint_release": (ctypes.c_int, [P]),
        "lbm_slab_exchange": (ctypes.c_int, [P, P]),
        "lbm_slab_message_bytes": (ctypes.c_long, [P]),
        "lbm_slab_pack": (ctypes.c_int, [P, ctypes.c_int, P]),
        "lbm_slab_unpack": (ctypes.c_int, [P, ctypes.c_int, P]),
        "lbm_city_generate": (ctypes.c_int, [ctypes.POINTER(LbmCityParams), c_float_p, ctypes.c_int,
                                             c_int_p, c_double_p]),
        "lbm_stl_write": (ctypes.c_int, [ctypes.c_char_p, c_float_p, ctypes.c_int]),
        "lbm_voxelize": (ctypes.c_int, [ctypes.POINTER(LbmConfig), c_float_p, ctypes.c_int] + [ctypes.c_double] * 4
                         + [c_uint8_p, ctypes.c_long, c_int_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
# NLOS_LBM_CHECK=1 loads the bounds-checked build instead of the product
CHECKED = os.environ.get("NLOS_LBM_CHECK", "0") not in ("", "0")
LIB_PATH = os.path.join(PACKAGE_DIR, "liblbm_b200_check.so" if CHECKED else "liblbm_b200.so")
