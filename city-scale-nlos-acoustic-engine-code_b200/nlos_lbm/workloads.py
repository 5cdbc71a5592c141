"""Seeded synthetic workloads at full size.

Lattice units throughout (dx = 1, c_phys = cs, so dt = 1 and times count
steps).  The city workloads stand in for the reference's real-city STL
(csx_model_binary.stl, 06:1131), which is not distributed: buildings are
seeded axis-aligned boxes written as triangles and voxelised by the
reference's heightmap ray cast.

  scatter    128^3 open box, rigid 16^3 cube, Gaussian pulse, 20-cell sponge
  lloyd      256x128x128, ground wall, moving sine source (Mach 0.1), trilinear
  city256    256x256x128 city patch with city1024's physics, 4 Ricker sources,
             64 probes, 4000 steps (its FP64 oracle series is a test fixture)
  city512    512x512x128 city (profiler-sized), 2 Ricker sources, 64 probes
  city1024   1024x1024x256 city, 4 Ricker sources at street level, 256 probes
  city2048   2048x2048x256 city, one source flying at z = 120 at Mach 0.15,
             512 probes (FP16 deviation storage, scale F16_HEADROOM/amplitude)
  adjoint256 256x256x128 city patch, tau 0.52, true source at street level
             emitting a Ricker wavelet (period 30 steps), 64 street-level
             receivers, 3000 steps; the trial source (the unknown of the
             localisation) sits a few cells away
  adjoint128 the same at 128x128x128 (profiler-sized: 160 MB per population
             buffer, still larger than L2)
  lloyd_a    02_lloyds_mirror.cpp at its own size (scheme A): 500x500x300 at
             dx 0.2, ground layer SOLID, tau ramp 0.51 -> 1, time-harmonic
             Gaussian source at the origin, 391 steps (to T = 45 s)
  doppler_a  03_doppler_effect.cpp at its own size (scheme A): 400x400x600 at
             dx 0.25, Mach 0.2 flow along z, zero-gradient halos, tau ramp
             0.51 -> 0.9 over 20 cells, 762 steps (to T = 110 s)
  scattering_a  01_acoustic_scattering.cpp at its own size (scheme A):
             320x320x8 at dx 0.05, cylinder of radius 0.5, initial pulse,
             destination blend sponge 0.5 deep, periodic z, 402 steps (to
             T = 11 s plus 01's 20 extra steps)
  hpc_a      04_hpc_scalability.cpp (the reference's MLUPS benchmark) at its
             own size (scheme A): 208^3 at dx 0.125, cylinder of radius 4,
             radial blend layer beyond r = 10, sine line source added before
             each step, periodic z, 2000 timed steps after 100
"""
import numpy as np

from . import abi

ALL_FACES = (1 << 6) - 1
# FP16 storage scale = F16_HEADROOM / source amplitude.  Probes far from a
# source see density deviations about 1e-3 of its amplitude; at a scale of
# 1/amplitude their populations fall into FP16's subnormal range (the 128^3
# scattering box over its 2000 steps: probe rel-L2 3.1e-3 against the FP64
# oracle).  A hundred times more keeps them normal (2.4e-4) and still leaves
# the stored values a factor ~650 below FP16's largest for peaks above the
# source amplitude.
F16_HEADROOM = 100.0
FIVE_FACES = ALL_FACES & ~(1 << abi.FACE_ZLO)
MACH_TO_CELLS = abi.CS   # cells/step per unit Mach (c = cs in lattice units)


# grid, default storage and description of the city workloads, known without
# building their geometry (bench.py's reference arm reports the headline
# workload's configuration without loading the library)
CITY_SUMMARY = {
    "city2048": ((2048, 2048, 256), "fp16", "synthetic city 2048x2048x256, source flying at z=120 Mach 0.15, "
                                            "512 probes"),
    "city1024": ((1024, 1024, 256), "fp32", "synthetic city 1024x1024x256, 4 Ricker sources, 256 street probes"),
    "city512": ((512, 512, 128), "fp32", "synthetic city 512x512x128, 2 Ricker sources, 64 street probes"),
    "city256": ((256, 256, 128), "fp32", "synthetic city patch 256x256x128, C3 physics, 4 Ricker sources, "
                                         "64 street probes"),
}


def lattice_config(nx, ny, nz, tau, **kw):
    base = dict(x_min=0.0, x_max=float(nx), y_min=0.0, y_max=float(ny), z_min=0.0, z_max=float(nz), dx=1.0,
                c_phys=abi.CS, tau=tau, sky_z=1e30)
    base.update(kw)
    return abi.reference_config(**base)


def footprints(tris):
    b = np.asarray(tris, dtype=np.float64).reshape(-1, 12, 3, 3)
    return b.min(axis=(1, 2)), b.max(axis=(1, 2))


def street_points(tris, nx, ny, n, z, seed, margin=40, clearance=2.0):
    """n random points at height z that lie in the streets (outside every
    building footprint by `clearance` cells) and `margin` cells inside the plan."""
    lo, hi = footprints(tris)
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        c = np.stack([rng.uniform(margin, nx - margin, 4 * n), rng.uniform(margin, ny - margin, 4 * n)], 1)
        inside = ((c[:, None, 0] > lo[None, :, 0] - clearance) & (c[:, None, 0] < hi[None, :, 0] + clearance)
                  & (c[:, None, 1] > lo[None, :, 1] - clearance) & (c[:, None, 1] < hi[None, :, 1] + clearance))
        ok = c[~inside.any(1)]
        out.extend(ok.tolist())
    pts = np.array(out[:n])
    return np.concatenate([pts, np.full((n, 1), z)], 1)


def city(nx, ny, nz, seed, storage, tau=0.51, sponge=32):
    from .solver import city_triangles

    tris, cov = city_triangles(nx, ny, seed=seed, fp=(20, 60), height=(10, 80), coverage=0.40, street=8,
                               margin=sponge + 8)
    amp = 1e-3
    cfg = lattice_config(nx, ny, nz, tau, sponge_width=float(sponge), sponge_faces=FIVE_FACES, storage=storage,
                         f16_scale=F16_HEADROOM / amp)
    return cfg, tris, cov, amp


def build(name, storage=None, seed=2024):
    """dict(cfg, sources, probes, triangles, steps, description)."""
    if name == "scatter":
        n = 128
        cfg = lattice_config(n, n, n, 0.55, face_bc=(abi.LBM_BC_NSCBC,) * 6, sponge_faces=ALL_FACES,
                             sponge_width=20.0, sponge_strength=0.5,
                             storage=abi.LBM_STORE_F32 if storage is None else storage,
                             f16_scale=F16_HEADROOM / 1e-3)
        c = n / 2
        tris = _cube(c - 8, c + 8)
        src = abi.reference_source(sx=c - 24 + 0.5, sy=c + 0.5, sz=c + 0.5, ex=c - 24 + 0.5, ey=c + 0.5,
                                   ez=c + 0.5, amp=1e-3, t0=40.0, sigma_t=8.0)
        a = 2 * np.pi * np.arange(8) / 8
        probes = np.stack([c + 40 * np.cos(a), c + 40 * np.sin(a), np.full(8, c)], 1)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=2000,
                    description="acoustic scattering 128^3, cube 16^3, Gaussian pulse")
    if name == "lloyd":
        cfg = lattice_config(256, 128, 128, 0.52, sponge_width=16.0, sponge_faces=FIVE_FACES,
                             storage=abi.LBM_STORE_F32 if storage is None else storage,
                             f16_scale=F16_HEADROOM / 5e-4)
        v = 0.1 * MACH_TO_CELLS
        src = abi.reference_source(sx=40.0, sy=64.0, sz=20.0, ex=250.0, ey=64.0, ez=20.0, speed=v, amp=5e-4,
                                   freq=1 / 50.0, waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_TRILINEAR)
        probes = np.stack([np.linspace(8.5, 247.5, 64), np.full(64, 64.5), np.full(64, 10.5)], 1)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, steps=6000,
                    description="Lloyd's mirror 256x128x128, moving sine source Mach 0.1, trilinear")
    if name == "city1024":
        st = abi.LBM_STORE_F32 if storage is None else storage
        cfg, tris, cov, amp = city(1024, 1024, 256, seed, st)
        pts = street_points(tris, 1024, 1024, 4 + 256, 2.5, seed)
        srcs = [abi.reference_source(sx=p[0], sy=p[1], sz=p[2], ex=p[0], ey=p[1], ez=p[2], amp=amp, freq=1 / 40.0,
                                     t0=60.0, waveform=abi.LBM_WAVE_RICKER, injection=abi.LBM_INJECT_TRILINEAR)
                for p in pts[:4]]
        return dict(cfg=cfg, sources=srcs, probes=pts[4:], triangles=tris, steps=4000, coverage=cov,
                    description=CITY_SUMMARY["city1024"][2])
    if name == "city256":
        # C3's physics on a 256x256x128 patch (tau 0.51, 32-cell sponge on the
        # sides and top, ground bounce-back, 4 Ricker sources at street
        # level, street-level probes) for its full 4000 steps: small enough
        # for the FP64 oracle to run its whole length on the host
        st = abi.LBM_STORE_F32 if storage is None else storage
        cfg, tris, cov, amp = city(256, 256, 128, seed, st)
        pts = street_points(tris, 256, 256, 4 + 64, 2.5, seed)
        srcs = [abi.reference_source(sx=p[0], sy=p[1], sz=p[2], ex=p[0], ey=p[1], ez=p[2], amp=amp, freq=1 / 40.0,
                                     t0=60.0, waveform=abi.LBM_WAVE_RICKER, injection=abi.LBM_INJECT_TRILINEAR)
                for p in pts[:4]]
        return dict(cfg=cfg, sources=srcs, probes=pts[4:], triangles=tris, steps=4000, coverage=cov,
                    description=CITY_SUMMARY["city256"][2])
    if name == "city512":
        # a few-GB version of the city for profiler captures
        st = abi.LBM_STORE_F32 if storage is None else storage
        cfg, tris, cov, amp = city(512, 512, 128, seed, st)
        pts = street_points(tris, 512, 512, 2 + 64, 2.5, seed)
        srcs = [abi.reference_source(sx=p[0], sy=p[1], sz=p[2], ex=p[0], ey=p[1], ez=p[2], amp=amp, freq=1 / 40.0,
                                     t0=60.0, waveform=abi.LBM_WAVE_RICKER, injection=abi.LBM_INJECT_TRILINEAR)
                for p in pts[:2]]
        return dict(cfg=cfg, sources=srcs, probes=pts[2:], triangles=tris, steps=4000, coverage=cov,
                    description=CITY_SUMMARY["city512"][2])
    if name == "city2048":
        st = abi.LBM_STORE_F16 if storage is None else storage
        cfg, tris, cov, amp = city(2048, 2048, 256, seed, st)
        probes = street_points(tris, 2048, 2048, 512, 2.5, seed)
        v = 0.15 * MACH_TO_CELLS
        src = abi.reference_source(sx=400.0, sy=600.0, sz=120.0, ex=1650.0, ey=1450.0, ez=120.0, speed=v, amp=amp,
                                   freq=1 / 40.0, waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_TRILINEAR)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=4000, coverage=cov,
                    description=CITY_SUMMARY["city2048"][2])
    if name in ("adjoint256", "adjoint128"):
        from .solver import city_triangles

        nx, ny, nz = (256, 256, 128) if name == "adjoint256" else (128, 128, 128)
        tris, cov = city_triangles(nx, ny, seed=seed, fp=(20, 60), height=(10, 80), coverage=0.40, street=8,
                                   margin=24)
        cfg = lattice_config(nx, ny, nz, 0.52, sponge_width=16.0, sponge_faces=FIVE_FACES,
                             storage=abi.LBM_STORE_F32 if storage is None else storage)
        pts = street_points(tris, nx, ny, 1 + 64, 2.5, seed, margin=24, clearance=3.0)
        true_xyz = pts[0] + np.array([0.0, 0.0, 1.1])
        trial_xyz = true_xyz + np.array([2.37, -1.61, 0.83])

        def ricker(x):
            return abi.reference_source(sx=x[0], sy=x[1], sz=x[2], ex=x[0], ey=x[1], ez=x[2], amp=1e-3,
                                        freq=1 / 30.0, t0=45.0, waveform=abi.LBM_WAVE_RICKER,
                                        injection=abi.LBM_INJECT_TRILINEAR)
        return dict(cfg=cfg, sources=[ricker(trial_xyz)], true_source=ricker(true_xyz), probes=pts[1:],
                    triangles=tris, steps=3000, coverage=cov,
                    description=f"transient localisation {nx}x{ny}x{nz} city patch, Ricker period 30, 64 receivers, "
                                "3000 steps")
    if name in ("lloyd_a", "lloyd_a_small"):
        # 02:53-56 domain, 02:32 dx, 02:126 omega, 02:138-181 physics; the
        # small one (profiler-sized) at dx 0.4: 250x250x150
        dx = 0.2 if name == "lloyd_a" else 0.4
        nx, nz = int(100.0 / dx + 0.5), int(60.0 / dx + 0.5)
        cfg = lattice_config(nx, nx, nz, 0.51, x_min=-50.0, x_max=50.0, y_min=-50.0, y_max=50.0, z_min=-10.0,
                             z_max=50.0, dx=dx, c_phys=1.0, face_bc=(abi.LBM_BC_REST,) * 6,
                             sponge_faces=ALL_FACES & ~(1 << abi.FACE_ZLO), sponge_width=15.0,
                             scheme=abi.LBM_SCHEME_A, tau_sponge_max=1.0, dt=0.577350269 * dx)
        mask = np.zeros((nz + 2, nx + 2, nx + 2), np.uint8)
        mask[1] = 1                                   # gz == 0 is SOLID (02:153-158)
        src = abi.reference_source(sx=0.0, sy=0.0, sz=0.0, ex=0.0, ey=0.0, ez=0.0, amp=0.5, freq=1.0 / 30.0,
                                   waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_FIELD,
                                   sigma_cells=np.sqrt(2.0 / (2.0 * np.log(2.0))) / dx,
                                   field_mode=abi.LBM_FIELD_DST)
        probes = np.stack([np.full(64, 0.1), np.linspace(-49.9, 49.9, 64), np.full(64, 0.1)], 1)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, mask=mask.ravel(), steps=391,
                    description=f"Lloyd's mirror (02) {nx}x{nx}x{nz}, scheme A, ground layer, tau ramp")
    if name == "doppler_a":
        # 03:32, 03:51, 03:55-63, 03:121, 03:135-169
        dx, Ma, cs = 0.25, 0.2, 0.5773502691896257
        n = (400, 400, 600)
        cfg = lattice_config(*n, 0.51, x_max=n[0] * dx, y_max=n[1] * dx, z_max=n[2] * dx, dx=dx, c_phys=1.0,
                             face_bc=(abi.LBM_BC_COPY,) * 6, sponge_faces=ALL_FACES, sponge_width=20.0,
                             scheme=abi.LBM_SCHEME_A, tau_sponge_max=0.9, flow=(0.0, 0.0, Ma * cs), dt=cs * dx)
        ctr = [(m / 2.0 + 0.5) * dx for m in n]
        src = abi.reference_source(sx=ctr[0], sy=ctr[1], sz=ctr[2], ex=ctr[0], ey=ctr[1], ez=ctr[2], amp=0.01,
                                   freq=1.0 / (30.0 * cs * dx), waveform=abi.LBM_WAVE_SINE,
                                   injection=abi.LBM_INJECT_FIELD, sigma_cells=1.0, field_mode=abi.LBM_FIELD_FORCE)
        probes = np.stack([np.full(64, ctr[0]), np.full(64, ctr[1]), np.linspace(1.0, n[2] * dx - 1.0, 64)], 1)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, mask=None, steps=762,
                    description="Doppler (03) 400x400x600, scheme A, Mach 0.2 flow, zero-gradient halos")
    if name == "scattering_a":
        # 01:54-56 domain, 01:65 dx, 01:67 pulse amplitude, 01:157-225 set-up, 01:486-488 steps
        dx, lo, hi = 0.05, -8.0, 8.0
        n = int((hi - lo) / dx + 0.5)
        nz = max(int(0.4 / dx + 0.5), 3)
        faces = (1 << abi.FACE_XLO) | (1 << abi.FACE_XHI) | (1 << abi.FACE_YLO) | (1 << abi.FACE_YHI)
        cfg = lattice_config(n, n, nz, 0.505, x_min=lo, x_max=hi, y_min=lo, y_max=hi, z_min=-0.2, z_max=0.2, dx=dx,
                             c_phys=1.0, face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2,
                             sponge_faces=faces, sponge_width=0.5 / dx, sponge_strength=1.0, sponge_blend=1,
                             scheme=abi.LBM_SCHEME_A, dt=np.sqrt(1.0 / 3.0) * dx)
        c = lo + (np.arange(-1, n + 1) + 0.5) * dx
        solid = (c[None, :] ** 2 + c[:, None] ** 2) < 0.25
        mask = np.broadcast_to(solid, (nz + 2,) + solid.shape).astype(np.uint8)
        pulse = 0.01 * np.exp(-np.log(2.0) * ((c[None, :] - 4.0) ** 2 + c[:, None] ** 2))
        pulse[solid] = 0.0
        rho0 = np.broadcast_to(pulse[1:-1, 1:-1], (nz, n, n))
        cell = lambda v: lo + (np.floor((v - lo) / dx) + 0.5) * dx
        r135 = np.deg2rad(135.0)
        probes = np.array([(cell(x), cell(y), -0.2 + (nz // 2 + 0.5) * dx)
                           for x, y in ((0.0, 1.0), (np.cos(r135), np.sin(r135)), (-1.0, 0.0))])
        max_steps = int(11.0 / (np.sqrt(1.0 / 3.0) * dx)) + 20
        return dict(cfg=cfg, sources=[], probes=probes, triangles=None, mask=np.ascontiguousarray(mask).ravel(),
                    rho0=np.ascontiguousarray(rho0).ravel(), steps=max_steps + 1,
                    description=f"acoustic scattering (01) {n}x{n}x{nz}, scheme A, cylinder, blend sponge, "
                                "periodic z")
    if name == "hpc_a":
        # 04:21-26, 04:52-54, 04:65-71, 04:177-235, 04:301, 04:360-404
        dx, half = 0.125, 13.0
        n = int(2 * half / dx + 0.5)
        cfg = lattice_config(n, n, n, 0.51, x_min=-half, x_max=half, y_min=-half, y_max=half, z_min=-half,
                             z_max=half, dx=dx, c_phys=1.0,
                             face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2, sponge_faces=0,
                             sponge_width=0.0, sponge_blend=1, scheme=abi.LBM_SCHEME_A, dt=0.577350269 * dx)
        solid, blend, weight = hpc_columns(dx, -half, n)
        mask = np.broadcast_to(solid, (n + 2,) + solid.shape).astype(np.uint8)
        src = abi.reference_source(sx=0.0, sy=-6.0, sz=0.0, ex=0.0, ey=-6.0, ez=0.0, amp=0.01, freq=1.0 / 30.0,
                                   waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_FIELD, sigma_cells=1.0,
                                   field_mode=abi.LBM_FIELD_PRE)
        zc = -half + (n // 2 + 0.5) * dx
        probes = np.array([[-half + (np.floor((px + half) / dx) + 0.5) * dx,
                            -half + (np.floor((py + half) / dx) + 0.5) * dx, zc]
                           for px, py in ((0.0, 7.0), (7.0, 0.0), (-7.0, 0.0), (0.0, -9.0))])
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, mask=np.ascontiguousarray(mask).ravel(),
                    blend_xy=blend.ravel(), field_xy=weight.ravel(), steps=2000,
                    description=f"scalability benchmark (04) {n}^3, scheme A, cylinder, radial blend layer, line "
                                "source, periodic z")
    raise KeyError(name)


def hpc_columns(dx, lo=-13.0, n=None, cyl_r=4.0, r0=10.0, th=3.0, strength=0.5, src_y=-6.0, b=2.0):
    """04_hpc_scalability.cpp's z-invariant set-up on an n x n column grid
    from lo at dx, with 04's own cell-centre expression lo + g dx + dx/2
    (04:187-188): SOLID cylinder r < cyl_r (04:191-194), radial blend layer
    0.5 min((r - 10)/3, 1)^2 beyond r = 10 (04:198-203), line-source weights
    exp(-ln2 d^2 / b) for d^2 = x^2 + (y - src_y)^2 <= 36 (04:220-224).
    Returns (solid[n+2, n+2] halo-inclusive, blend[n, n], weight[n, n])."""
    g = np.arange(-1, n + 1)
    c = lo + g * dx + 0.5 * dx
    x, y = c[None, :], c[:, None]
    r = np.sqrt(x * x + y * y)
    solid = r < cyl_r
    ratio = np.minimum((r - r0) / th, 1.0)
    blend = np.where(~solid & (r > r0), strength * ratio * ratio, 0.0)
    d2 = x * x + (y - src_y) * (y - src_y)
    weight = np.where(d2 > 36.0, 0.0, np.exp(-np.log(2.0) * d2 / b))
    return solid, blend[1:-1, 1:-1], weight[1:-1, 1:-1]


def _cube(a, b):
    v = [(a, a, a), (b, a, a), (b, b, a), (a, b, a), (a, a, b), (b, a, b), (b, b, b), (a, b, b)]
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
    out = []
    for q in quads:
        out.append(v[q[0]] + v[q[1]] + v[q[2]])
        out.append(v[q[0]] + v[q[2]] + v[q[3]])
    return np.asarray(out, dtype=np.float32)


def cells(cfg):
    nx = int((cfg.x_max - cfg.x_min) / cfg.dx + 0.5)
    ny = int((cfg.y_max - cfg.y_min) / cfg.dx + 0.5)
    nz = int((cfg.z_max - cfg.z_min) / cfg.dx + 0.5)
    return nx, ny, nz
