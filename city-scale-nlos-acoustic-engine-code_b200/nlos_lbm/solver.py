"""Python mirror of the reference solver interface over the C-ABI.

``LBMSolver`` has the public fields and methods of the reference's
``LBMSolver`` (06_transient_localization_dx1.cpp:241-1122): the scenario is
set through fields, ``init()`` voxelises and uploads, and the step methods
``apply_source(t)``, ``exchange_halos()``, ``step_collision_bgk()`` and
``run(T_total, Frames)`` advance it.  ``Solver`` is the lower-level handle
wrapper the tests and the benchmark use.  Every call goes through
liblbm_b200.so; there is no Python or CPU fallback: a missing library or GPU
raises.
"""
import ctypes
import os
import warnings

import numpy as np

from . import abi


class LBMError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None


def library():
    """The loaded liblbm_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(abi.LIB_PATH):
            raise ImportError(f"{abi.LIB_PATH} is missing: build it with `python -m nlos_lbm.build` "
                              "(there is no CPU fallback)")
        _lib = abi.bind_product(ctypes.CDLL(abi.LIB_PATH))
    return _lib


def _ptr(a, t=abi.c_double_p):
    return a.ctypes.data_as(t)


class Solver:
    """One solver handle: config + geometry + sources + probes -> device state."""

    def __init__(self, cfg, sources=(), probes=None, triangles=None, stl=None, stl_offset=(0.0, 0.0, 0.0),
                 mask=None, blend_xy=None, field_xy=None):
        self.lib = library()
        self.cfg = cfg
        h = ctypes.c_void_p()
        st = self.lib.lbm_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise LBMError(st, "lbm_create: " + self.lib.lbm_status_string(st).decode())
        self.h = h
        self.warnings = []
        if stl is not None:
            st = self.lib.lbm_set_geometry_stl(self.h, stl.encode(), 1.0, *stl_offset)
            self._check(st, "lbm_set_geometry_stl")
        elif triangles is not None:
            t = np.ascontiguousarray(triangles, dtype=np.float32).reshape(-1, 9)
            self._check(self.lib.lbm_set_geometry_triangles(self.h, _ptr(t, abi.c_float_p), len(t), 1.0,
                                                            *stl_offset), "lbm_set_geometry_triangles")
        if mask is not None:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            nx = int(round((cfg.x_max - cfg.x_min) / cfg.dx)) + 2
            ny = int(round((cfg.y_max - cfg.y_min) / cfg.dx)) + 2
            nz = int(round((cfg.z_max - cfg.z_min) / cfg.dx)) + 2
            self._check(self.lib.lbm_set_mask(self.h, _ptr(m, abi.c_uint8_p), nx, ny, nz), "lbm_set_mask")
        # scheme A: per-column blend strengths and source weights (nx*ny, x fastest)
        for arr, fn, what in ((blend_xy, self.lib.lbm_set_blend_xy, "lbm_set_blend_xy"),
                              (field_xy, self.lib.lbm_set_field_weights_xy, "lbm_set_field_weights_xy")):
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
                self._check(fn(self.h, _ptr(a), a.size), what)
        for s in sources:
            self._check(self.lib.lbm_add_source(self.h, ctypes.byref(s)), "lbm_add_source")
        self.nprobe = 0
        if probes is not None:
            p = np.ascontiguousarray(probes, dtype=np.float64).reshape(-1, 3)
            self.nprobe = len(p)
            self._check(self.lib.lbm_set_probes(self.h, _ptr(p), len(p)), "lbm_set_probes")
        self.init_status = self._check(self.lib.lbm_init(self.h), "lbm_init")
        n3, nh = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        self._check(self.lib.lbm_get_dims(self.h, n3, nh), "lbm_get_dims")
        self.dims, self.dims_halo = tuple(n3), tuple(nh)
        self.dt = self.lib.lbm_get_dt(self.h)

    def _check(self, st, what):
        if st < 0:
            msg = self.lib.lbm_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise LBMError(st, f"{what}: {self.lib.lbm_status_string(st).decode()} {msg}".strip())
        if st > 0:
            self.warnings.append(st)
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def ncell_halo(self):
        nx, ny, nz = self.dims_halo
        return nx * ny * nz

    # -- stepping (06:576-972, 06:1077-1092)
    def step(self, n=1):
        self._check(self.lib.lbm_step(self.h, int(n)), "lbm_step")

    def apply_source(self, t):
        self._check(self.lib.lbm_apply_source(self.h, float(t)), "lbm_apply_source")

    def exchange_halos(self):
        self._check(self.lib.lbm_exchange_halos(self.h), "lbm_exchange_halos")

    def step_collision_bgk(self):
        self._check(self.lib.lbm_step_collision_bgk(self.h), "lbm_step_collision_bgk")

    def record_probes(self):
        self._check(self.lib.lbm_record_probes(self.h), "lbm_record_probes")

    def run(self, T_total, frames=1):
        self._check(self.lib.lbm_run(self.h, float(T_total), int(frames)), "lbm_run")

    def synchronize(self):
        self._check(self.lib.lbm_synchronize(self.h), "lbm_synchronize")

    @property
    def step_count(self):
        return int(self.lib.lbm_get_step(self.h))

    # -- results
    def get_probes(self):
        n = ctypes.c_long()
        self._check(self.lib.lbm_get_probes(self.h, None, 0, ctypes.byref(n)), "lbm_get_probes")
        out = np.empty(max(n.value * self.nprobe, 1))
        self._check(self.lib.lbm_get_probes(self.h, _ptr(out), out.size, ctypes.byref(n)), "lbm_get_probes")
        return out[: n.value * self.nprobe].reshape(n.value, self.nprobe)

    def get_probe_energy(self):
        out = np.empty(max(self.nprobe, 1))
        self._check(self.lib.lbm_get_probe_energy(self.h, _ptr(out)), "lbm_get_probe_energy")
        return out[: self.nprobe]

    def probe_info(self):
        owned = np.zeros(max(self.nprobe, 1), dtype=np.int32)
        solid = np.zeros(max(self.nprobe, 1), dtype=np.int32)
        self._check(self.lib.lbm_probe_info(self.h, _ptr(owned, abi.c_int_p), _ptr(solid, abi.c_int_p)),
                    "lbm_probe_info")
        return owned[: self.nprobe].astype(bool), solid[: self.nprobe].astype(bool)

    def get_f(self):
        out = np.empty(self.ncell_halo * 19)
        self._check(self.lib.lbm_get_f(self.h, _ptr(out), out.size), "lbm_get_f")
        return out

    def set_f(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._check(self.lib.lbm_set_f(self.h, _ptr(f), f.size), "lbm_set_f")

    def set_density(self, rho_prime):
        """Scheme A: start at rest with density 1 + rho' at every interior
        fluid cell (nx*ny*nz values, x fastest), before the first step."""
        r = np.ascontiguousarray(rho_prime, dtype=np.float64).ravel()
        self._check(self.lib.lbm_set_density(self.h, _ptr(r), r.size), "lbm_set_density")

    def get_rho(self):
        nx, ny, nz = self.dims
        out = np.empty(nx * ny * nz, dtype=np.float32)
        self._check(self.lib.lbm_get_rho(self.h, _ptr(out, abi.c_float_p), out.size), "lbm_get_rho")
        return out.reshape(nz, ny, nx)

    def get_mask(self):
        out = np.empty(self.ncell_halo, dtype=np.uint8)
        self._check(self.lib.lbm_get_mask(self.h, _ptr(out, abi.c_uint8_p), out.size), "lbm_get_mask")
        return out

    # -- measurement
    def set_kernel_timing(self, on):
        self._check(self.lib.lbm_set_kernel_timing(self.h, int(bool(on))), "lbm_set_kernel_timing")

    def kernel_time(self):
        ms, n = ctypes.c_double(), ctypes.c_long()
        self._check(self.lib.lbm_get_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(n)), "lbm_get_kernel_time")
        return ms.value, n.value

    @property
    def launch_count(self):
        return int(self.lib.lbm_get_launch_count(self.h))

    @property
    def bytes_per_cell(self):
        return int(self.lib.lbm_bytes_per_cell(self.h))

    @property
    def stream(self):
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self.lib.lbm_get_stream(self.h) or 0)

    def transfer_bytes(self):
        h2d, d2h = ctypes.c_long(), ctypes.c_long()
        self._check(self.lib.lbm_get_transfer_bytes(self.h, ctypes.byref(h2d), ctypes.byref(d2h)),
                    "lbm_get_transfer_bytes")
        return h2d.value, d2h.value

    # -- adjoint
    def adjoint_grad(self, observed, ckpt_outer=0, ckpt_inner=0):
        """Misfit and its gradient for the probe series `observed` [nsteps, nprobe]
        (lbm_adjoint_grad): returns (loss, grad_pos[3], grad_signal[nsteps],
        predicted[nsteps, nprobe]).  The solver is left at the rest state."""
        obs = np.ascontiguousarray(observed, dtype=np.float64)
        if obs.ndim != 2 or obs.shape[1] != self.nprobe:
            raise ValueError("observed must be [nsteps, nprobe]")
        T = obs.shape[0]
        loss = ctypes.c_double()
        gpos = np.zeros(3)
        gsig = np.zeros(T)
        pred = np.zeros((T, self.nprobe))
        self._check(self.lib.lbm_adjoint_grad(self.h, T, _ptr(obs), int(ckpt_outer), int(ckpt_inner),
                                              ctypes.byref(loss), _ptr(gpos), _ptr(gsig), _ptr(pred)),
                    "lbm_adjoint_grad")
        return loss.value, gpos, gsig, pred

    def adjoint_plan(self, nsteps, ckpt_outer=0, ckpt_inner=0):
        """(outer, inner, device_bytes, forward_steps) of lbm_adjoint_plan."""
        o, i = ctypes.c_int(), ctypes.c_int()
        b, f = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.lbm_adjoint_plan(self.h, int(nsteps), int(ckpt_outer), int(ckpt_inner), ctypes.byref(o),
                                              ctypes.byref(i), ctypes.byref(b), ctypes.byref(f)), "lbm_adjoint_plan")
        return o.value, i.value, b.value, f.value

    def adjoint_release(self):
        """Frees the adjoint workspace kept by the handle (lbm_adjoint_release)."""
        self._check(self.lib.lbm_adjoint_release(self.h), "lbm_adjoint_release")

    def check_status(self):
        """(site, index) of the first failed bounds check since the last call
        (site 0: none); bounds-checked library only (NLOS_LBM_CHECK=1)."""
        site, index = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.lbm_check_status(self.h, ctypes.byref(site), ctypes.byref(index)), "lbm_check_status")
        return site.value, index.value

    def check_selftest(self):
        """Fails one bounds check on purpose (bounds-checked library only)."""
        self._check(self.lib.lbm_check_selftest(self.h), "lbm_check_selftest")

    def clear_sources(self):
        self._check(self.lib.lbm_clear_sources(self.h), "lbm_clear_sources")

    def add_source(self, src):
        self._check(self.lib.lbm_add_source(self.h, ctypes.byref(src)), "lbm_add_source")


class SlabGroup:
    """One grid split into z-slabs, one handle each (on `devices`, default all
    on the configured device), stepped with the reference's loop body per slab
    and one lbm_slab_exchange per cut between the halo fill and the collision:
    the split run reproduces the undivided run.  Probes and fields are merged
    back into whole-grid form."""

    def __init__(self, cfg, nslabs, sources=(), probes=None, triangles=None, stl=None, stl_offset=(0.0, 0.0, 0.0),
                 devices=None, cuts=None):
        nz = int((cfg.z_max - cfg.z_min) / cfg.dx + 0.5)
        if cuts is None:
            cuts = [round(i * nz / nslabs) for i in range(1, nslabs)]
        bounds = [0] + list(cuts) + [nz]
        self.bounds = bounds
        self.slabs = []
        for i in range(len(bounds) - 1):
            c = abi.LbmConfig.from_buffer_copy(cfg)
            c.slab_k0, c.slab_nz = bounds[i], bounds[i + 1] - bounds[i]
            if devices is not None:
                c.device = devices[i % len(devices)]
            self.slabs.append(Solver(c, sources, probes, triangles=triangles, stl=stl, stl_offset=stl_offset))
        self.lib = self.slabs[0].lib
        self.dt = self.slabs[0].dt
        self.nprobe = self.slabs[0].nprobe
        self.steps = 0

    def step(self, n=1):
        for _ in range(int(n)):
            t = self.steps * self.dt
            for s in self.slabs:
                s.apply_source(t)
                s.exchange_halos()
            for lo, hi in zip(self.slabs[:-1], self.slabs[1:]):
                lo._check(self.lib.lbm_slab_exchange(lo.h, hi.h), "lbm_slab_exchange")
            for s in self.slabs:
                s.step_collision_bgk()
                s.record_probes()
            self.steps += 1

    def get_probes(self):
        """[step][probe]: each probe from the slab that holds its cell (NaN outside the grid)."""
        out = None
        for s in self.slabs:
            p = s.get_probes()
            out = p.copy() if out is None else np.where(np.isnan(out), p, out)
        return out

    def get_rho(self):
        return np.concatenate([s.get_rho() for s in self.slabs], axis=0)

    def close(self):
        for s in self.slabs:
            s.close()


def city_triangles(nx, ny, seed, dx=1.0, fp=(20, 60), height=(10, 80), coverage=0.40, street=8, margin=0):
    """Seeded synthetic city (lbm_city_generate): float32 [ntri, 9] and the plan coverage."""
    lib = library()
    p = abi.LbmCityParams(nx, ny, dx, seed, fp[0], fp[1], height[0], height[1], coverage, street, margin)
    n = ctypes.c_int()
    cov = ctypes.c_double()
    st = lib.lbm_city_generate(ctypes.byref(p), None, 0, ctypes.byref(n), ctypes.byref(cov))
    if st not in (0, abi.LBM_ERR_CAPACITY):
        raise LBMError(st, "lbm_city_generate")
    out = np.empty((max(n.value, 1), 9), dtype=np.float32)
    st = lib.lbm_city_generate(ctypes.byref(p), _ptr(out, abi.c_float_p), n.value, ctypes.byref(n), ctypes.byref(cov))
    if st != 0:
        raise LBMError(st, "lbm_city_generate")
    return out[: n.value], cov.value


def voxelize(cfg, triangles=None, stl_offset=(0.0, 0.0, 0.0)):
    """Host voxeliser (lbm_voxelize): the uint8 mask lbm_init would build, reference layout."""
    lib = library()
    t = np.ascontiguousarray(triangles if triangles is not None else np.zeros((0, 9)), dtype=np.float32).reshape(-1, 9)
    n3 = (ctypes.c_int * 3)()
    st = lib.lbm_voxelize(ctypes.byref(cfg), _ptr(t, abi.c_float_p), len(t), 1.0, *stl_offset, None, 0, n3)
    if st not in (0, abi.LBM_ERR_CAPACITY):
        raise LBMError(st, "lbm_voxelize")
    out = np.empty(n3[0] * n3[1] * n3[2], dtype=np.uint8)
    st = lib.lbm_voxelize(ctypes.byref(cfg), _ptr(t, abi.c_float_p), len(t), 1.0, *stl_offset,
                          _ptr(out, abi.c_uint8_p), out.size, n3)
    if st != 0:
        raise LBMError(st, "lbm_voxelize")
    return out


def stl_write(path, tris):
    t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    st = library().lbm_stl_write(path.encode(), _ptr(t, abi.c_float_p), len(t))
    if st != 0:
        raise LBMError(st, "lbm_stl_write")


class DroneSource:
    """DroneSource (06:211-239): straight flight from (sx,sy,sz) to (ex,ey,ez)."""

    def __init__(self):
        self.sx = self.sy = self.sz = 0.0
        self.ex = self.ey = self.ez = 0.0
        self.speed = 0.0
        self.amp = 0.0
        self.freq = 0.0


class Probe:
    def __init__(self, name, x, y, z):
        self.name, self.x, self.y, self.z = name, float(x), float(y), float(z)
        self.p_history = []


class LBMSolver:
    """Field-for-field mirror of the reference LBMSolver (06:241-268) on the GPU.

    ``waveform`` selects the source time function: "gauss" (06:579-581) or
    "sine" (08:543).  Extra knobs of this library (storage, face types,
    sponge) are read from ``config`` when given.
    """

    def __init__(self, waveform="gauss"):
        self.stl_file = ""
        self.stl_sx = self.stl_sy = self.stl_sz = 0.0
        self.drone = DroneSource()
        self.use_geometry = True
        self.X_MIN, self.X_MAX = 0.0, 1650.0
        self.Y_MIN, self.Y_MAX = 0.0, 1150.0
        self.Z_MIN, self.Z_MAX = 0.0, 250.0
        self.DX = 2.0
        self.output_world_coords = True
        self.probes = []
        self.tau = 0.55
        self.use_nscbc = True
        self.waveform = waveform
        self.config = None
        self.solver = None

    def init(self, argc=0, argv=None):
        cfg = self.config or abi.reference_config()
        cfg.x_min, cfg.x_max = self.X_MIN, self.X_MAX
        cfg.y_min, cfg.y_max = self.Y_MIN, self.Y_MAX
        cfg.z_min, cfg.z_max = self.Z_MIN, self.Z_MAX
        cfg.dx, cfg.tau = self.DX, self.tau
        cfg.use_geometry = int(self.use_geometry)
        if not self.use_nscbc:
            for f in range(6):
                if cfg.face_bc[f] == abi.LBM_BC_NSCBC:
                    cfg.face_bc[f] = abi.LBM_BC_REST
        d = self.drone
        src = abi.reference_source(sx=d.sx, sy=d.sy, sz=d.sz, ex=d.ex, ey=d.ey, ez=d.ez, speed=d.speed,
                                   amp=d.amp, freq=d.freq,
                                   waveform=abi.LBM_WAVE_SINE if self.waveform == "sine" else abi.LBM_WAVE_GAUSS)
        probes = np.array([[p.x, p.y, p.z] for p in self.probes]) if self.probes else None
        self.solver = Solver(cfg, [src], probes,
                             stl=self.stl_file if self.use_geometry else None,
                             stl_offset=(self.stl_sx, self.stl_sy, self.stl_sz))
        if abi.LBM_WARN_STL_NOT_LOADED in self.solver.warnings:
            print("Warning: STL not loaded, using empty geometry.")   # 06:409
        if self.probes:
            _, solid = self.solver.probe_info()
            for p, s in zip(self.probes, solid):
                if s:
                    print(f"WARNING: Probe {p.name} is trapped inside SOLID building!")   # 06:434
        self._recorded = 0

    def apply_source(self, t):
        self.solver.apply_source(t)

    def exchange_halos(self):
        self.solver.exchange_halos()

    def step_collision_bgk(self):
        self.solver.step_collision_bgk()

    def _sync_probes(self):
        if not self.probes:
            return
        series = self.solver.get_probes()
        owned, _ = self.solver.probe_info()
        for k, p in enumerate(self.probes):
            if owned[k]:
                p.p_history = list(series[:, k])

    def run(self, T_total, Frames):
        self.solver.run(T_total, Frames)
        self._sync_probes()

    def write_vtk(self, path):
        """Legacy-VTK structured-points file of (float)(rho-1) (06:975-1062),
        binary big-endian float32 instead of ASCII."""
        rho = self.solver.get_rho()
        nz, ny, nx = rho.shape
        ox, oy, oz = self.X_MIN, self.Y_MIN, self.Z_MIN
        if self.output_world_coords:
            ox, oy, oz = ox - self.stl_sx, oy - self.stl_sy, oz - self.stl_sz
        with open(path, "wb") as fh:
            fh.write(b"# vtk DataFile Version 3.0\nLBM Urban Acoustics\nBINARY\nDATASET STRUCTURED_POINTS\n")
            fh.write(f"DIMENSIONS {nx} {ny} {nz}\nORIGIN {ox} {oy} {oz}\n".encode())
            fh.write(f"SPACING {self.DX} {self.DX} {self.DX}\nPOINT_DATA {nx * ny * nz}\n".encode())
            fh.write(b"SCALARS PressureAmp float 1\nLOOKUP_TABLE default\n")
            fh.write(rho.astype(">f4").tobytes())
