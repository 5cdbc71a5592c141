"""Oracle bindings -- TEST INFRASTRUCTURE ONLY.

Two CPU checkers for the D3Q19 acoustic step, loaded through ctypes:

* ``OracleSolver`` -- the FP64 C restatement (oracle/lbm_oracle.c), built by
  ``make -C oracle`` into oracle/_build/liblbm_oracle.so.
* ``RefSolver`` -- the unmodified reference solver (06 or 08) through the
  include harness (oracle/ref_harness.cpp), built by ``make -C oracle ref``
  into oracle/_ref/.  Present only where the reference sources were available
  at build time.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package; the product library never calls it.
"""
import ctypes
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200"))
from nlos_lbm import abi  # noqa: E402  (ctypes ABI description only)

ORACLE_LIB = os.path.join(HERE, "_build", "liblbm_oracle.so")
REF_LIBS = {"06": os.path.join(HERE, "_ref", "libref06.so"), "08": os.path.join(HERE, "_ref", "libref08.so")}

_dp = abi.c_double_p
_lib = None


def reference_dir():
    """Directory of the reference sources: NLOS_REFERENCE_DIR, else the
    default written in oracle/Makefile."""
    r = subprocess.run(["make", "-s", "-C", HERE, "print-ref-dir"], check=True, capture_output=True, text=True)
    return r.stdout.strip()


def build(ref=False):
    """Compile the restatement (and the reference harness when ref=True)."""
    cmd = ["make", "-s", "-C", HERE, "all"] + (["ref"] if ref else [])
    subprocess.run(cmd, check=True)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        lib = ctypes.CDLL(ORACLE_LIB)
        P = ctypes.c_void_p
        sig = {
            "orc_create": (P, [ctypes.POINTER(abi.LbmConfig)]),
            "orc_destroy": (None, [P]),
            "orc_set_geometry_triangles": (ctypes.c_int, [P, abi.c_float_p, ctypes.c_int] + [ctypes.c_double] * 4),
            "orc_set_geometry_stl": (ctypes.c_int, [P, ctypes.c_char_p] + [ctypes.c_double] * 4),
            "orc_set_mask": (ctypes.c_int, [P, abi.c_uint8_p]),
            "orc_add_source": (ctypes.c_int, [P, ctypes.POINTER(abi.LbmSource)]),
            "orc_set_probes": (ctypes.c_int, [P, _dp, ctypes.c_int]),
            "orc_init": (ctypes.c_int, [P]),
            "orc_apply_source": (None, [P, ctypes.c_double]),
            "orc_exchange_halos": (None, [P]),
            "orc_step_collision_bgk": (None, [P]),
            "orc_record_probes": (None, [P]),
            "orc_step": (None, [P, ctypes.c_int]),
            "orc_set_threads": (None, [ctypes.c_int]),
            "orc_get_dims": (None, [P, abi.c_int_p, abi.c_int_p]),
            "orc_get_dt": (ctypes.c_double, [P]),
            "orc_get_f": (None, [P, _dp]),
            "orc_set_f": (None, [P, _dp]),
            "orc_set_density": (None, [P, _dp]),
            "orc_set_blend_xy": (ctypes.c_int, [P, _dp]),
            "orc_set_field_xy": (ctypes.c_int, [P, _dp]),
            "orc_get_mask": (None, [P, abi.c_uint8_p]),
            "orc_get_rho": (None, [P, _dp]),
            "orc_get_sponge": (None, [P, _dp]),
            "orc_get_ground_height": (None, [P, _dp]),
            "orc_get_probes": (ctypes.c_long, [P, _dp, ctypes.c_long]),
            "orc_adjoint_grad": (ctypes.c_int, [P, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, _dp]),
            "orc_get_tau_a": (None, [P, _dp]),
        }
        for n, (r, a) in sig.items():
            fn = getattr(lib, n)
            fn.restype, fn.argtypes = r, a
        _lib = lib
    return _lib


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def box_triangles(boxes):
    """Axis-aligned boxes (x0, y0, z0, x1, y1, z1) -> float32 [n*12, 9] triangles."""
    out = []
    for (x0, y0, z0, x1, y1, z1) in boxes:
        v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
             (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
        quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
        for a, b, c, d in quads:
            out.append(v[a] + v[b] + v[c])
            out.append(v[a] + v[c] + v[d])
    return np.asarray(out, dtype=np.float32).reshape(-1, 9)


def write_stl(path, tris):
    """Binary STL in the layout GeometryEngine::load reads (06:49-58, 06:70-111)."""
    tris = np.asarray(tris, dtype=np.float32).reshape(-1, 9)
    with open(path, "wb") as fh:
        fh.write(b"oracle test geometry".ljust(80, b"\0"))
        fh.write(struct.pack("<I", len(tris)))
        for t in tris:
            a, b, c = t[0:3].astype(np.float64), t[3:6].astype(np.float64), t[6:9].astype(np.float64)
            n = np.cross(b - a, c - a)
            ln = np.linalg.norm(n)
            n = (n / ln if ln > 0 else n).astype(np.float32)
            fh.write(n.tobytes() + t.tobytes() + b"\0\0")


class OracleSolver:
    """FP64 restatement with the same call surface as the reference LBMSolver."""

    def __init__(self, cfg, sources=(), probes=None, triangles=None, stl=None, stl_offset=(0.0, 0.0, 0.0),
                 mask=None, threads=None, blend_xy=None, field_xy=None):
        self.lib = _load()
        if threads:
            self.lib.orc_set_threads(int(threads))
        self.cfg = cfg
        self.h = self.lib.orc_create(ctypes.byref(cfg))
        self._keep = []
        for arr, fn in ((blend_xy, self.lib.orc_set_blend_xy), (field_xy, self.lib.orc_set_field_xy)):
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
                fn(self.h, _ptr(a))
        if stl is not None:
            self.stl_status = self.lib.orc_set_geometry_stl(self.h, stl.encode(), 1.0, *stl_offset)
        elif triangles is not None:
            t = np.ascontiguousarray(triangles, dtype=np.float32)
            self.lib.orc_set_geometry_triangles(self.h, _ptr(t, abi.c_float_p), len(t), 1.0, *stl_offset)
        for s in sources:
            self.lib.orc_add_source(self.h, ctypes.byref(s))
        self.nprobe = 0
        if probes is not None:
            p = np.ascontiguousarray(probes, dtype=np.float64).reshape(-1, 3)
            self.nprobe = len(p)
            self.lib.orc_set_probes(self.h, _ptr(p), len(p))
        self.init_status = self.lib.orc_init(self.h)
        if mask is not None:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            self.lib.orc_set_mask(self.h, _ptr(m, abi.c_uint8_p))
            self.init_status = self.lib.orc_init(self.h)
        n3, nh = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        self.lib.orc_get_dims(self.h, n3, nh)
        self.dims, self.dims_halo = tuple(n3), tuple(nh)
        self.dt = self.lib.orc_get_dt(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def ncell_halo(self):
        nx, ny, nz = self.dims_halo
        return nx * ny * nz

    def step(self, n=1):
        self.lib.orc_step(self.h, int(n))

    def apply_source(self, t):
        self.lib.orc_apply_source(self.h, t)

    def exchange_halos(self):
        self.lib.orc_exchange_halos(self.h)

    def step_collision_bgk(self):
        self.lib.orc_step_collision_bgk(self.h)

    def record_probes(self):
        self.lib.orc_record_probes(self.h)

    def get_f(self):
        out = np.empty(self.ncell_halo * 19)
        self.lib.orc_get_f(self.h, _ptr(out))
        return out

    def set_f(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self.lib.orc_set_f(self.h, _ptr(f))

    def set_density(self, rho_prime):
        """Scheme A: rest state with density 1 + rho' at interior fluid cells (x fastest)."""
        r = np.ascontiguousarray(rho_prime, dtype=np.float64).ravel()
        self.lib.orc_set_density(self.h, _ptr(r))

    def get_mask(self):
        out = np.empty(self.ncell_halo, dtype=np.uint8)
        self.lib.orc_get_mask(self.h, _ptr(out, abi.c_uint8_p))
        return out

    def get_rho(self):
        out = np.empty(self.ncell_halo)
        self.lib.orc_get_rho(self.h, _ptr(out))
        return out

    def get_sponge(self):
        out = np.empty(self.ncell_halo)
        self.lib.orc_get_sponge(self.h, _ptr(out))
        return out

    def get_ground_height(self):
        nx, ny, _ = self.dims_halo
        out = np.empty(nx * ny)
        self.lib.orc_get_ground_height(self.h, _ptr(out))
        return out

    def get_tau_a(self):
        """Per-cell tau of a scheme-A run (the ramp sponge)."""
        out = np.empty(self.ncell_halo)
        self.lib.orc_get_tau_a(self.h, _ptr(out))
        return out

    def adjoint_grad(self, observed, K=0):
        """FP64 discrete adjoint (orc_adjoint_grad): (loss, grad_pos[3],
        grad_signal[nsteps], predicted[nsteps, nprobe]); needs the state right
        after construction and restores it."""
        obs = np.ascontiguousarray(observed, dtype=np.float64)
        T = obs.shape[0]
        loss = ctypes.c_double()
        gpos, gsig, pred = np.zeros(3), np.zeros(T), np.zeros((T, self.nprobe))
        st = self.lib.orc_adjoint_grad(self.h, T, _ptr(obs), int(K), ctypes.byref(loss), _ptr(gpos), _ptr(gsig),
                                       _ptr(pred))
        if st != 0:
            raise RuntimeError("orc_adjoint_grad failed: %d" % st)
        return loss.value, gpos, gsig, pred

    def get_probes(self):
        cap = 1
        while True:
            out = np.empty(max(cap, 1))
            n = self.lib.orc_get_probes(self.h, _ptr(out), cap)
            if n >= 0:
                return out[: n * self.nprobe].reshape(n, self.nprobe)
            cap = cap * 4 + 1024 * max(self.nprobe, 1)


class RefAParams(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in "x_min x_max y_min y_max z_min z_max dx amp b_param omega Ma "
                 "tau_bulk tau_sponge_max".split()] + [("sponge_width", ctypes.c_int), ("omega_lb", ctypes.c_double)])


def refa_available(which):
    return os.path.exists(os.path.join(HERE, "_ref", "libref%s.so" % which))


class RefASolver:
    """An unmodified family-A reference program (01 acoustic scattering, 02
    Lloyd's mirror, 03 Doppler or 04 scalability benchmark) through
    oracle/ref_harness_a.cpp: set-up, then steps of [apply_source() (04)] +
    exchange_halos() + step(); fields in the reference's own layout."""

    def __init__(self, which, **params):
        lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libref%s.so" % which))
        P = ctypes.c_void_p
        for n, (r, a) in {"refa_create": (P, [ctypes.POINTER(RefAParams)]), "refa_destroy": (None, [P]),
                          "refa_dims": (None, [P, abi.c_int_p]), "refa_dt": (ctypes.c_double, [P]),
                          "refa_step": (None, [P, ctypes.c_int]), "refa_get_rho": (None, [P, _dp]),
                          "refa_get_f": (None, [P, _dp]), "refa_get_tau": (None, [P, _dp]),
                          "refa_get_source": (None, [P, _dp]), "refa_get_mask": (None, [P, abi.c_uint8_p]),
                          "refa_get_sponge": (None, [P, _dp]),
                          "refa_set_threads": (None, [ctypes.c_int])}.items():
            fn = getattr(lib, n)
            fn.restype, fn.argtypes = r, a
        self.lib = lib
        p = RefAParams()
        for k, v in params.items():
            setattr(p, k, v)
        self.h = lib.refa_create(ctypes.byref(p))
        n3 = (ctypes.c_int * 3)()
        lib.refa_dims(self.h, n3)
        self.dims_halo = tuple(n3)
        self.dt = lib.refa_dt(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.refa_destroy(self.h)
            self.h = None

    @property
    def ncell_halo(self):
        nx, ny, nz = self.dims_halo
        return nx * ny * nz

    def step(self, n=1):
        self.lib.refa_step(self.h, int(n))

    def _get(self, fn, n, dtype=np.float64, t=_dp):
        out = np.empty(n, dtype=dtype)
        fn(self.h, _ptr(out, t))
        return out

    def get_rho(self):
        return self._get(self.lib.refa_get_rho, self.ncell_halo)

    def get_f(self):
        return self._get(self.lib.refa_get_f, self.ncell_halo * 19)

    def get_tau(self):
        return self._get(self.lib.refa_get_tau, self.ncell_halo)

    def get_source(self):
        return self._get(self.lib.refa_get_source, self.ncell_halo)

    def get_mask(self):
        return self._get(self.lib.refa_get_mask, self.ncell_halo, np.uint8, abi.c_uint8_p)

    def get_sponge(self):
        """01's destination-blend sponge strengths (zeros for 02 and 03)."""
        return self._get(self.lib.refa_get_sponge, self.ncell_halo)


class RefParams(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in "x_min x_max y_min y_max z_min z_max dx tau".split()]
                + [("use_geometry", ctypes.c_int), ("use_nscbc", ctypes.c_int), ("stl_file", ctypes.c_char_p)]
                + [(n, ctypes.c_double) for n in
                   "stl_sx stl_sy stl_sz d_sx d_sy d_sz d_ex d_ey d_ez d_speed d_amp d_freq".split()]
                + [("n_probes", ctypes.c_int), ("probe_xyz", _dp)])


def ref_available(which="06"):
    return os.path.exists(REF_LIBS[which])


class RefSolver:
    """The unmodified reference LBMSolver (06: Gaussian pulse, 08: sine) via
    the include harness.  Supports exactly the reference's own options."""

    def __init__(self, which, x_range, y_range, z_range, dx, tau, drone, probes=None, stl=None,
                 stl_offset=(0.0, 0.0, 0.0), use_geometry=None, use_nscbc=True, threads=None):
        path = REF_LIBS[which]
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run make -C oracle ref with the reference sources present)")
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        lib.ref_create.restype, lib.ref_create.argtypes = P, [ctypes.POINTER(RefParams)]
        for n in ("ref_destroy", "ref_exchange_halos", "ref_step_collision_bgk", "ref_record_probes"):
            getattr(lib, n).restype, getattr(lib, n).argtypes = None, [P]
        lib.ref_apply_source.restype, lib.ref_apply_source.argtypes = None, [P, ctypes.c_double]
        lib.ref_run_steps.restype, lib.ref_run_steps.argtypes = None, [P, ctypes.c_int, ctypes.c_int]
        lib.ref_dims.restype, lib.ref_dims.argtypes = None, [P, abi.c_int_p]
        lib.ref_dt.restype, lib.ref_dt.argtypes = ctypes.c_double, [P]
        for n in ("ref_get_f", "ref_set_f", "ref_get_rho", "ref_get_sponge"):
            getattr(lib, n).restype, getattr(lib, n).argtypes = None, [P, _dp]
        lib.ref_get_mask.restype, lib.ref_get_mask.argtypes = None, [P, abi.c_uint8_p]
        lib.ref_get_probes.restype, lib.ref_get_probes.argtypes = ctypes.c_int, [P, _dp, ctypes.c_long]
        lib.ref_set_threads.restype, lib.ref_set_threads.argtypes = None, [ctypes.c_int]
        self.lib = lib
        if threads:
            lib.ref_set_threads(int(threads))
        pr = np.ascontiguousarray(probes if probes is not None else np.zeros((0, 3)), dtype=np.float64).reshape(-1, 3)
        self._probes = pr
        self.nprobe = len(pr)
        self._stl = (stl or "").encode()
        p = RefParams()
        p.x_min, p.x_max = x_range
        p.y_min, p.y_max = y_range
        p.z_min, p.z_max = z_range
        p.dx, p.tau = dx, tau
        p.use_geometry = int(stl is not None) if use_geometry is None else int(use_geometry)
        p.use_nscbc = int(use_nscbc)
        p.stl_file = self._stl
        p.stl_sx, p.stl_sy, p.stl_sz = stl_offset
        (p.d_sx, p.d_sy, p.d_sz, p.d_ex, p.d_ey, p.d_ez, p.d_speed, p.d_amp, p.d_freq) = drone
        p.n_probes = self.nprobe
        p.probe_xyz = _ptr(pr)
        self.h = lib.ref_create(ctypes.byref(p))
        d = (ctypes.c_int * 3)()
        lib.ref_dims(self.h, d)
        self.dims_halo = tuple(d)
        self.dt = lib.ref_dt(self.h)
        self.step_index = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    @property
    def ncell_halo(self):
        nx, ny, nz = self.dims_halo
        return nx * ny * nz

    def step(self, n=1):
        self.lib.ref_run_steps(self.h, self.step_index, int(n))
        self.step_index += int(n)

    def get_f(self):
        out = np.empty(self.ncell_halo * 19)
        self.lib.ref_get_f(self.h, _ptr(out))
        return out

    def get_mask(self):
        out = np.empty(self.ncell_halo, dtype=np.uint8)
        self.lib.ref_get_mask(self.h, _ptr(out, abi.c_uint8_p))
        return out

    def get_rho(self):
        out = np.empty(self.ncell_halo)
        self.lib.ref_get_rho(self.h, _ptr(out))
        return out

    def get_sponge(self):
        out = np.empty(self.ncell_halo)
        self.lib.ref_get_sponge(self.h, _ptr(out))
        return out

    def get_probes(self):
        cap = max(1, (self.step_index + 1) * max(self.nprobe, 1))
        out = np.empty(cap)
        n = self.lib.ref_get_probes(self.h, _ptr(out), cap)
        return out[: n * self.nprobe].reshape(n, self.nprobe)
