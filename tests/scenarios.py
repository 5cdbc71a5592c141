"""Seeded parity scenarios shared by the GPU tests, the fixture generator and
the smoke check.  Each scenario is a small version of one workload the solver
is run on (reference-native set-ups of 06/08 and reduced versions of the
scattering / Lloyd's-mirror / synthetic-city workloads); both the CUDA solver
and the FP64 oracle are built from the same description.
"""
import numpy as np

from nlos_lbm import abi, workloads

ALL_FACES = (1 << 6) - 1
FIVE_FACES = ALL_FACES & ~(1 << abi.FACE_ZLO)


def boxes_to_triangles(boxes):
    from oracle import box_triangles

    return box_triangles(boxes)


def lattice_config(nx, ny, nz, tau, **kw):
    """Lattice units: dx = 1 and c_phys = cs, so dt = 1 and t counts steps."""
    base = dict(x_min=0.0, x_max=float(nx), y_min=0.0, y_max=float(ny), z_min=0.0, z_max=float(nz), dx=1.0,
                c_phys=abi.CS, tau=tau, sky_z=1e30)
    base.update(kw)
    return abi.reference_config(**base)


def ring_probes(center, radius, n, z):
    a = 2 * np.pi * np.arange(n) / n
    return np.stack([center[0] + radius * np.cos(a), center[1] + radius * np.sin(a), np.full(n, z)], 1)


def scenario(name, storage=abi.LBM_STORE_F32, f16_scale=1.0):
    """Returns dict(cfg, sources, probes, triangles, steps)."""
    if name == "ref06_box":
        # 06 physics: physical units, dx = 1 m, Gaussian pulse (06:579-581), ground wall,
        # NSCBC on the other faces, 20-cell sponge at strength 0.35.
        cfg = abi.reference_config(x_min=0, x_max=48, y_min=0, y_max=32, z_min=0, z_max=30, dx=1.0, tau=0.55)
        src = abi.reference_source(sx=24.3, sy=16.2, sz=12.7, ex=24.3, ey=16.2, ez=12.7, amp=10.0)
        tris = boxes_to_triangles([(10, 8, 0, 22, 20, 12), (30, 5, 0, 41, 14, 7), (26, 20, 0, 38, 30, 16)])
        probes = np.array([[20.5, 16.5, 10.5], [30.5, 16.5, 20.5], [5.2, 3.3, 2.1], [15.0, 12.0, 5.0]])
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=80)
    if name == "ref08_moving":
        # 08 physics: sine source flying across the domain (08:543, 06:221-238).
        cfg = abi.reference_config(x_min=0, x_max=48, y_min=0, y_max=32, z_min=0, z_max=30, dx=1.0, tau=0.55)
        src = abi.reference_source(sx=5.0, sy=6.0, sz=20.0, ex=40.0, ey=25.0, ez=22.0, speed=300.0, amp=0.5,
                                   freq=20.0, waveform=abi.LBM_WAVE_SINE)
        tris = boxes_to_triangles([(10, 8, 0, 22, 20, 12), (30, 5, 0, 41, 14, 7)])
        probes = np.array([[20.5, 16.5, 14.5], [40.5, 26.5, 20.5], [8.0, 28.0, 3.0]])
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=60)
    if name == "scatter_small":
        # Acoustic scattering: open box (NSCBC on all six faces), rigid cube at the
        # centre, Gaussian pulse 12 cells away, sponge on every face ramping to 0.5.
        n = 48
        cfg = lattice_config(n, n, n, 0.55, face_bc=(abi.LBM_BC_NSCBC,) * 6, sponge_faces=ALL_FACES,
                             sponge_width=10.0, sponge_strength=0.5, storage=storage, f16_scale=f16_scale)
        c = n / 2
        tris = boxes_to_triangles([(c - 4, c - 4, c - 4, c + 4, c + 4, c + 4)])
        src = abi.reference_source(sx=c - 12.0 + 0.3, sy=c + 0.2, sz=c + 0.1, ex=c - 11.7, ey=c + 0.2, ez=c + 0.1,
                                   amp=1e-3, t0=20.0, sigma_t=4.0)
        probes = ring_probes((c, c), 16.0, 8, c)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=240)
    if name == "lloyd_small":
        # Lloyd's mirror: ground wall, moving sine source, trilinear injection, probe line.
        cfg = lattice_config(64, 32, 32, 0.52, sponge_width=8.0, sponge_faces=FIVE_FACES, storage=storage,
                             f16_scale=f16_scale)
        src = abi.reference_source(sx=12.0, sy=16.0, sz=10.0, ex=60.0, ey=16.0, ez=10.0, speed=0.0577, amp=5e-4,
                                   freq=1.0 / 50.0, waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_TRILINEAR)
        probes = np.stack([np.linspace(4.5, 59.5, 16), np.full(16, 16.5), np.full(16, 5.5)], 1)
        return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, steps=300)
    if name == "city_small":
        # Synthetic city: seeded box buildings (STL triangles -> voxeliser), ground wall,
        # sponge on sides and top, two Ricker sources at street level.
        import nlos_lbm

        nx, ny, nz = 96, 80, 40
        tris, _ = nlos_lbm.city_triangles(nx, ny, seed=7, fp=(12, 24), height=(6, 30), street=6, margin=4)
        cfg = lattice_config(nx, ny, nz, 0.51, sponge_width=10.0, sponge_faces=FIVE_FACES, storage=storage,
                             f16_scale=f16_scale)
        mask = nlos_lbm.voxelize(cfg, tris).reshape(nz + 2, ny + 2, nx + 2)
        rng = np.random.default_rng(7)
        pts = []
        while len(pts) < 2 + 12:
            x, y = rng.uniform(6, nx - 6), rng.uniform(6, ny - 6)
            if mask[3, int(y) + 1, int(x) + 1] == 0:
                pts.append((x, y, 2.5))
        srcs = [abi.reference_source(sx=p[0], sy=p[1], sz=p[2], ex=p[0], ey=p[1], ez=p[2], amp=1e-3, freq=1 / 40.0,
                                     t0=40.0, waveform=abi.LBM_WAVE_RICKER, injection=abi.LBM_INJECT_TRILINEAR)
                for p in pts[:2]]
        probes = np.array(pts[2:])
        return dict(cfg=cfg, sources=srcs, probes=probes, triangles=tris, steps=200)
    raise KeyError(name)


def adjoint_scenario(nx=48, ny=40, nz=24, steps=160, injection=abi.LBM_INJECT_TRILINEAR, speed=0.0, nprobe=16,
                     seed=11):
    """Transient localisation on a synthetic-city patch (a reduced version of
    the 256x256x128, 3000-step case): a true source at street level emits a
    Ricker wavelet (period 30 steps); receivers at street level record it; the
    trial source sits 1-2 cells away.  Returns dict(cfg, true, trial, probes,
    triangles, steps, observed) with `observed` from the FP64 oracle."""
    import nlos_lbm
    from oracle import OracleSolver

    tris, _ = nlos_lbm.city_triangles(nx, ny, seed=seed, fp=(8, 14), height=(4, 16), street=5, margin=3)
    cfg = lattice_config(nx, ny, nz, 0.52, sponge_width=6.0, sponge_faces=FIVE_FACES)
    mask = nlos_lbm.voxelize(cfg, tris).reshape(nz + 2, ny + 2, nx + 2)
    rng = np.random.default_rng(seed)

    def street_point(z, used):
        while True:
            x, y = rng.uniform(5, nx - 5), rng.uniform(5, ny - 5)
            c = (int(x), int(y), int(z))
            ok = all(mask[c[2] + 1 + dz, c[1] + 1 + dy, c[0] + 1 + dx] == 0
                     for dx in (-2, -1, 0, 1, 2) for dy in (-2, -1, 0, 1, 2) for dz in (-1, 0, 1))
            if ok and c not in used:
                used.add(c)
                return x, y, z

    used = set()
    tx, ty, tz = street_point(3.6, used)
    # trial position: displaced, with fractional parts away from the trilinear cell edges
    px = np.floor(tx + 1.4) + 0.83
    py = np.floor(ty - 0.9) + 0.29
    pz = 4.12
    probes = np.array([street_point(rng.uniform(1.5, 6.5), used) for _ in range(nprobe)])

    def src(x, y, z):
        return abi.reference_source(sx=x, sy=y, sz=z, ex=x + (40.0 if speed else 0.0), ey=y, ez=z, speed=speed,
                                    amp=1e-3, freq=1.0 / 30.0, t0=30.0, waveform=abi.LBM_WAVE_RICKER,
                                    injection=injection, radius=2, sigma_cells=1.0)

    true_src, trial = src(tx, ty, tz), src(px, py, pz)
    o = OracleSolver(cfg, [true_src], probes, triangles=tris)
    o.step(steps)
    observed = o.get_probes()
    return dict(cfg=cfg, true=true_src, trial=trial, probes=probes, triangles=tris, steps=steps,
                observed=observed)


def source_copy(src, shift=(0.0, 0.0, 0.0), table=None):
    """Copy of an lbm_source with its path shifted rigidly by `shift` and,
    with `table`, the waveform replaced by that per-step signal (amp 1).
    The table array must outlive the source: it is returned alongside."""
    names = [f[0] for f in abi.LbmSource._fields_]
    kw = {n: getattr(src, n) for n in names if n not in ("table", "table_len")}
    for a, n in enumerate(("sx", "sy", "sz")):
        kw[n] += shift[a]
    for a, n in enumerate(("ex", "ey", "ez")):
        kw[n] += shift[a]
    keep = None
    if table is not None:
        keep = np.ascontiguousarray(table, dtype=np.float64)
        kw.update(waveform=abi.LBM_WAVE_TABLE, amp=1.0, table=keep.ctypes.data_as(abi.c_double_p),
                  table_len=len(keep))
    return abi.reference_source(**kw), keep


def source_signal(src, steps, dt):
    """val(t_s) of a Ricker source at steps 0..steps-1 (the forward's waveform)."""
    t = np.arange(steps) * dt
    a = (np.pi * src.freq * (t - src.t0)) ** 2
    return src.amp * (1.0 - 2.0 * a) * np.exp(-a)


def misfit(pred, observed):
    """1/2 sum (pred - observed)^2 over the probes inside the grid (FP64)."""
    m = np.isfinite(pred[0])
    return 0.5 * float(np.sum((pred[:, m] - observed[:, m]) ** 2))


def family_a(name, n=40, steps=60):
    """Reduced versions of the family-A programs for the scheme-A path.

    lloyd_a: 02_lloyds_mirror.cpp (Lloyd's mirror): x, y in [-4, 4], z in
    [-0.8, 4] at dx = 0.2 (02's cell size), the first layer above z_min SOLID
    (02:153-158), rest halos, tau 0.51 ramping to 1 over 15 cells from x-,
    x+, y-, y+, z+ (02:164-179), time-harmonic Gaussian source
    0.5 exp(-ln2 r^2 / 2) sin(pi t / 15) at the origin added at the
    destination (02:181, 02:373); dt = 0.577350269 dx / c (02:36).
    doppler_a: 03_doppler_effect.cpp (uniform flow): an n^3 grid at
    dx = 0.25, Mach 0.2 flow along z, zero-gradient halos, tau 0.51 ramping to
    0.9 over 10 cells from every face, Gaussian forcing 0.01 exp(-r^2 /
    (2 dx^2)) sin(2 pi s / 30) at the grid centre (03:121, 03:135-169).

    Returns dict(cfg, sources, probes, mask, steps, ref, ref_params)."""
    if name == "lloyd_a":
        dx = 0.2
        cfg = abi.reference_config(x_min=-4.0, x_max=4.0, y_min=-4.0, y_max=4.0, z_min=-0.8, z_max=4.0, dx=dx,
                                   c_phys=1.0, tau=0.51, use_geometry=0, face_bc=(abi.LBM_BC_REST,) * 6,
                                   sponge_faces=ALL_FACES & ~(1 << abi.FACE_ZLO), sponge_width=15.0, sky_z=1e30,
                                   scheme=abi.LBM_SCHEME_A, tau_sponge_max=1.0, dt=0.577350269 * dx / 1.0)
        nx, ny, nz = 40, 40, 24
        mask = np.zeros((nz + 2, ny + 2, nx + 2), np.uint8)
        mask[1] = 1                                  # gz == 0 is SOLID; halos stay FLUID
        sig_cells = np.sqrt(2.0 / (2.0 * np.log(2.0))) / dx   # exp(-ln2 r^2 / b), b = 2
        src = abi.reference_source(sx=0.0, sy=0.0, sz=0.0, ex=0.0, ey=0.0, ez=0.0, amp=0.5, freq=1.0 / 30.0,
                                   waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_FIELD,
                                   sigma_cells=sig_cells, field_mode=abi.LBM_FIELD_DST)
        tz = -0.8 + (int((0.0 + 0.8) / dx + 0.5) + 0.5) * dx
        probes = np.stack([np.full(8, 0.1), np.linspace(-3.5, 3.5, 8), np.full(8, tz)], 1)
        ref_params = dict(x_min=-4.0, x_max=4.0, y_min=-4.0, y_max=4.0, z_min=-0.8, z_max=4.0, dx=dx, amp=0.5,
                          b_param=2.0)
        return dict(cfg=cfg, sources=[src], probes=probes, mask=mask.ravel(), steps=steps, ref="02",
                    ref_params=ref_params)
    if name == "doppler_a":
        dx, Ma, cs = 0.25, 0.2, 0.5773502691896257
        dt = cs * dx / 1.0
        cfg = abi.reference_config(x_min=0.0, x_max=n * dx, y_min=0.0, y_max=n * dx, z_min=0.0, z_max=n * dx, dx=dx,
                                   c_phys=1.0, tau=0.51, use_geometry=0, face_bc=(abi.LBM_BC_COPY,) * 6,
                                   sponge_faces=ALL_FACES, sponge_width=10.0, sky_z=1e30, scheme=abi.LBM_SCHEME_A,
                                   tau_sponge_max=0.9, flow=(0.0, 0.0, Ma * cs), dt=dt)
        c = (n / 2.0 + 0.5) * dx                      # (g - n/2) dx about cell centres (03:135-168)
        src = abi.reference_source(sx=c, sy=c, sz=c, ex=c, ey=c, ez=c, amp=0.01,
                                   freq=(2.0 * np.pi / 30.0) / (2.0 * np.pi * dt), waveform=abi.LBM_WAVE_SINE,
                                   injection=abi.LBM_INJECT_FIELD, sigma_cells=1.0, field_mode=abi.LBM_FIELD_FORCE)
        probes = np.stack([np.full(8, c), np.full(8, c), np.linspace(1.1, n * dx - 1.1, 8)], 1)
        ref_params = dict(x_min=0.0, x_max=n * dx, y_min=0.0, y_max=n * dx, z_min=0.0, z_max=n * dx, dx=dx,
                          amp=0.01, Ma=Ma, tau_bulk=0.51, tau_sponge_max=0.9, sponge_width=10)
        return dict(cfg=cfg, sources=[src], probes=probes, mask=None, steps=steps, ref="03", ref_params=ref_params)
    if name == "scattering_a":
        return scattering_a(steps=steps)
    if name == "hpc_a":
        return hpc_a(steps=steps)
    raise KeyError(name)


def hpc_a(steps=40, dx=0.5, half=13.0):
    """04_hpc_scalability.cpp (the reference's scaling benchmark) on a reduced
    grid: [-13, 13]^3 at dx 0.5 instead of 0.125 (04:52-54, 04:21); tau 0.51
    (04:301); periodic z and rest x/y halos (04:51, 04:237-297); the radial
    blend layer and the line source of workloads.hpc_columns, a sine of amplitude 0.01
    and angular frequency pi/15 added before each step (04:65-67, 04:212-235);
    dt = 0.577350269 dx (04:22-26).  Probes at cell centres in the fluid."""
    n = int(2 * half / dx + 0.5)
    cfg = abi.reference_config(x_min=-half, x_max=half, y_min=-half, y_max=half, z_min=-half, z_max=half, dx=dx,
                               c_phys=1.0, tau=0.51, use_geometry=0,
                               face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2,
                               sponge_faces=0, sponge_width=0.0, sponge_blend=1, sky_z=1e30,
                               scheme=abi.LBM_SCHEME_A, tau_sponge_max=0.0, dt=0.577350269 * dx)
    solid, blend, weight = workloads.hpc_columns(dx, -half, n)
    mask = np.broadcast_to(solid, (n + 2,) + solid.shape).astype(np.uint8)
    src = abi.reference_source(sx=0.0, sy=-6.0, sz=0.0, ex=0.0, ey=-6.0, ez=0.0, amp=0.01, freq=1.0 / 30.0,
                               waveform=abi.LBM_WAVE_SINE, injection=abi.LBM_INJECT_FIELD, sigma_cells=1.0,
                               field_mode=abi.LBM_FIELD_PRE)
    cell = lambda v: -half + (np.floor((v + half) / dx) + 0.5) * dx
    pts = [(0.0, -6.0), (6.0, 0.0), (-6.0, 0.0), (0.0, 7.0), (9.0, 9.0)]
    zc = -half + (n // 2 + 0.5) * dx
    probes = np.array([(cell(px), cell(py), zc) for px, py in pts])
    ref_params = dict(x_min=-half, x_max=half, y_min=-half, y_max=half, z_min=-half, z_max=half, dx=dx, amp=0.01)
    return dict(cfg=cfg, sources=[src], probes=probes, mask=np.ascontiguousarray(mask).ravel(), blend_xy=blend.ravel(),
                field_xy=weight.ravel(), steps=steps, ref="04", ref_params=ref_params)


def scattering_a(steps=60, dx=0.1, x=(-3.0, 6.0), y=(-3.0, 3.0), z=(-0.2, 0.2), amp=0.01):
    """01_acoustic_scattering.cpp (pulse scattered by a cylinder) on a reduced
    domain: a cylinder of radius 0.5 at the origin along z (SOLID where
    x^2 + y^2 < 0.25 at cell centres, halos included, 01:167-185), an initial
    density pulse 1 + amp exp(-ln2 ((x-4)^2 + y^2)) at fluid cells
    (01:187-205), tau 0.505 everywhere (01:305), rest halos on x and y and
    periodic z (01:105-107), the destination blend sponge 0.5 deep on x and y
    with strength 1 (01:170-171, 01:207-225); dt = sqrt(1/3) dx / c (01:33-38).
    Probes sit at cell centres next to 01's A, B, C (01:157-162)."""
    nxg = int((x[1] - x[0]) / dx + 0.5)
    nyg = int((y[1] - y[0]) / dx + 0.5)
    nzg = max(int((z[1] - z[0]) / dx + 0.5), 3)
    faces = (1 << abi.FACE_XLO) | (1 << abi.FACE_XHI) | (1 << abi.FACE_YLO) | (1 << abi.FACE_YHI)
    cfg = abi.reference_config(x_min=x[0], x_max=x[1], y_min=y[0], y_max=y[1], z_min=z[0], z_max=z[1], dx=dx,
                               c_phys=1.0, tau=0.505, use_geometry=0,
                               face_bc=(abi.LBM_BC_REST,) * 4 + (abi.LBM_BC_PERIODIC,) * 2,
                               sponge_faces=faces, sponge_width=0.5 / dx, sponge_strength=1.0, sponge_blend=1,
                               sky_z=1e30, scheme=abi.LBM_SCHEME_A, tau_sponge_max=0.0,
                               dt=np.sqrt(1.0 / 3.0) * dx / 1.0)
    xc = x[0] + (np.arange(-1, nxg + 1) + 0.5) * dx
    yc = y[0] + (np.arange(-1, nyg + 1) + 0.5) * dx
    solid2 = (xc[None, :] ** 2 + yc[:, None] ** 2) < 0.25
    mask = np.broadcast_to(solid2, (nzg + 2,) + solid2.shape).astype(np.uint8)
    pulse2 = amp * np.exp(-np.log(2.0) * ((xc[None, :] - 4.0) ** 2 + yc[:, None] ** 2))
    pulse2[solid2] = 0.0
    rho0 = np.broadcast_to(pulse2[1:-1, 1:-1], (nzg, nyg, nxg)).copy()
    cell = lambda v, lo: lo + (np.floor((v - lo) / dx) + 0.5) * dx
    r135 = np.deg2rad(135.0)
    pts = [(0.0, 1.0), (np.cos(r135), np.sin(r135)), (-1.0, 0.0), (2.0, 0.0), (4.0, 0.0)]
    zc = z[0] + (nzg // 2 + 0.5) * dx
    probes = np.array([(cell(px, x[0]), cell(py, y[0]), zc) for px, py in pts])
    ref_params = dict(x_min=x[0], x_max=x[1], y_min=y[0], y_max=y[1], z_min=z[0], z_max=z[1], dx=dx, amp=amp)
    return dict(cfg=cfg, sources=[], probes=probes, mask=np.ascontiguousarray(mask).ravel(), rho0=rho0.ravel(),
                steps=steps, ref="01", ref_params=ref_params)


def build_pair(sc):
    """(CUDA solver, FP64 oracle) for one scenario."""
    from nlos_lbm import Solver
    from oracle import OracleSolver

    g = Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    o = OracleSolver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    return g, o


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
