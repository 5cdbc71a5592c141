"""Benchmark of the fused D3Q19 acoustic step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full time step of the synthetic-city workload (source
injection, open-boundary ghost fill, fused stream+bounce-back+BGK+sponge
kernel, probe sampling).  Headline workload: the 2048x2048x256 synthetic
city with FP16 deviation storage (1.07 G cells).  Also measured on one GPU:
FP32 and FP16 storage on the 1024x1024x256 city (the FP16/FP32 ratio) and the
end-to-end rate through the C-ABI with host buffers.  Multi-GPU runs are
independent replicas (one per rank, no data exchange), value = all ranks'
cell updates / the slowest rank's device time.

--impl reference times the reference solver's own CPU step
(06_transient_localization_dx1.cpp:576-972 via oracle/_ref, or the FP64
oracle port where the reference was not built) on a bounded sub-domain of the
same city with all host threads.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200"))
sys.path.insert(0, REPO)

METRIC = "D3Q19 GLUPS, %HBM peak: FP16-store vs FP32 @<=1e-3 probe L2; adjoint grad/s"
# bytes of DRAM traffic per cell update of the fused step kernel, from ncu
# captures of the default kernels on the 512x512x128 city (k_step_hw:
# 2.644e9 B, k_step<float>: 5.132e9 B for 33.55e6 cells)
NCU_TRAFFIC_PER_CELL = {"fp16": 2.644e9 / 33554432, "fp32": 5.132e9 / 33554432}
UNIT = "GLUPS"
DATA = "synthetic (seeded box city voxelised from STL triangles)"
L2_BYTES = 126e6   # B200 L2
# steps of the FP16-vs-FP32 probe comparison on the 1024x1024x256 city: the
# workload's whole configured length
ERR_STEPS = 4000


def headline_config(name, storage, n, dims=None, desc=None):
    """The `config` of both arms' lines: the workload, its grid and storage,
    the multi-GPU form and the L2 rule (known without building the city
    workloads; other workloads pass their grid and description)."""
    from nlos_lbm import workloads

    if name in workloads.CITY_SUMMARY:
        dims, default_storage, desc = workloads.CITY_SUMMARY[name]
    else:
        default_storage = "fp32"
    storage = storage or default_storage
    cells = dims[0] * dims[1] * dims[2]
    pop_bytes = cells * (76 if storage == "fp16" else 152)
    return {"workload": f"{name}: {desc}", "grid": list(dims), "storage": storage,
            "parallelism": f"replicas x{n}" if n > 1 else "single GPU",
            "l2": "inputs larger than L2" if pop_bytes > 2 * L2_BYTES else "inputs about the size of L2"}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------------------- our arm

def make_reducers(dist, device):
    """barrier() and reduce_max(x) over the ranks (identity without a process group)."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()

    def reduce_max(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, reduce_max


def replica_glups(world, cells, steps, ms_max):
    """Whole-job rate of `world` independent replicas: every rank updates
    cells x steps; the job takes as long as the slowest rank."""
    return world * cells * steps / (ms_max / 1e3) / 1e9


def make_solver(name, storage, device):
    import nlos_lbm
    from nlos_lbm import workloads

    w = workloads.build(name, storage=storage)
    w["cfg"].device = device
    t0 = time.time()
    s = nlos_lbm.Solver(w["cfg"], w["sources"], w["probes"], triangles=w["triangles"], mask=w.get("mask"),
                        blend_xy=w.get("blend_xy"), field_xy=w.get("field_xy"))
    if w.get("rho0") is not None:
        s.set_density(w["rho0"])
    return s, w, time.time() - t0


def device_timed_steps(solver, steps, torch, barrier):
    """Runs `steps` steps bracketed by CUDA events on the library's stream."""
    stream = torch.cuda.ExternalStream(solver.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    solver.synchronize()
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    solver.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    return e0.elapsed_time(e1)


def measure(name, storage, steps, warmup, device, torch, barrier, reduce_max, kernel_timing=True):
    from nlos_lbm import workloads

    s, w, setup_s = make_solver(name, storage, device)
    nx, ny, nz = workloads.cells(w["cfg"])
    ncell = nx * ny * nz
    # fluid share of the interior cells (GLUPS count every cell, SOLID ones included)
    solid = np.count_nonzero(s.get_mask().reshape(nz + 2, ny + 2, nx + 2)[1:-1, 1:-1, 1:-1])
    fluid_fraction = 1.0 - solid / ncell
    s.step(warmup)
    # the timed steps run as the library runs them (CUDA graphs); the step
    # kernel's own duration comes from as many further steps with per-launch
    # events (which replace the graphs by direct launches)
    l0 = s.launch_count
    ms = device_timed_steps(s, steps, torch, barrier)
    launches = s.launch_count - l0
    kms, kn = 0.0, 0
    if kernel_timing:
        s.set_kernel_timing(True)
        s.step(steps)
        kms, kn = s.kernel_time()
        s.set_kernel_timing(False)
    ms_max = reduce_max(ms)
    probes = s.get_probes()
    res = dict(name=name, storage="fp16" if s.bytes_per_cell == 76 else "fp32", cells=ncell, dims=[nx, ny, nz],
               steps=steps, ms=ms_max, ms_local=ms, setup_s=setup_s, glups_rank=ncell * steps / (ms_max / 1e3) / 1e9,
               kernel_ms_avg=kms / max(kn, 1), kernel_launches=kn, launches=launches,
               bytes_per_cell=s.bytes_per_cell, probes_finite=bool(np.all(np.isfinite(probes))),
               description=w["description"], coverage=w.get("coverage"), fluid_fraction=fluid_fraction,
               f16_scale=w["cfg"].f16_scale if s.bytes_per_cell == 76 else None)
    return s, w, res


def e2e_measure(solver, w, steps):
    """Through the C-ABI with host buffers: the source amplitude series goes
    host->device (lbm_add_source with a table waveform, uploaded inside
    lbm_step) and the probe series device->host (lbm_get_probes).  A workload
    without a source (01's initial pulse) has only the probe series."""
    import ctypes

    from nlos_lbm import abi

    if not w["sources"]:
        solver.get_probes()
        h0, d0 = solver.transfer_bytes()
        t0 = time.perf_counter()
        solver.step(steps)
        series = solver.get_probes()
        t1 = time.perf_counter()
        h1, d1 = solver.transfer_bytes()
        assert series.shape[0] >= steps
        return (t1 - t0) * 1e3, (h1 - h0) / steps, (d1 - d0) / steps
    base = w["sources"][0]
    s0 = solver.step_count
    table = np.zeros(s0 + steps)
    t = np.arange(s0, s0 + steps, dtype=np.float64)
    table[s0:] = np.sin(2 * np.pi * t / 40.0)
    solver.get_probes()   # drain earlier rows
    h0, d0 = solver.transfer_bytes()
    t0 = time.perf_counter()
    solver.clear_sources()
    src = abi.LbmSource()
    ctypes.pointer(src)[0] = base   # every field of the workload's source, then a table waveform
    src.waveform = abi.LBM_WAVE_TABLE
    src.table = table.ctypes.data_as(abi.c_double_p)
    src.table_len = len(table)
    solver.add_source(src)
    solver.step(steps)
    series = solver.get_probes()
    t1 = time.perf_counter()
    h1, d1 = solver.transfer_bytes()
    assert series.shape[0] >= steps
    return (t1 - t0) * 1e3, (h1 - h0) / steps, (d1 - d0) / steps


def adjoint_measure(device, torch, reps=2, ckpt=(200, 0), workload="adjoint256", steps=None):
    """Gradients per second of lbm_adjoint_grad on the 256x256x128 patch
    (3000 steps, 64 receivers): observed series from a forward run of the
    true source, then the misfit gradient at the trial source, timed with CUDA
    events on the library's stream around whole lbm_adjoint_grad calls
    (median of `reps`; the untimed warm-up call allocates the workspace the
    handle keeps)."""
    import nlos_lbm
    from nlos_lbm import workloads

    w = workloads.build(workload)
    if steps:
        w["steps"] = int(steps)
    w["cfg"].device = device
    truth = nlos_lbm.Solver(w["cfg"], [w["true_source"]], w["probes"], triangles=w["triangles"])
    truth.step(w["steps"])
    observed = truth.get_probes()
    truth.close()
    s = nlos_lbm.Solver(w["cfg"], w["sources"], w["probes"], triangles=w["triangles"])
    k_outer, k_inner, dev_bytes, fwd_steps = s.adjoint_plan(w["steps"], *ckpt)
    stream = torch.cuda.ExternalStream(s.stream)
    s.adjoint_grad(observed, *ckpt)   # warm-up: workspace allocation, first launches
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = s.launch_count
        e0.record(stream)
        loss, gpos, gsig, _ = s.adjoint_grad(observed, *ckpt)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        launches = s.launch_count - l0
    nx, ny, nz = workloads.cells(w["cfg"])
    ms = float(np.median(times))
    return {"workload": workload + ": " + w["description"], "grad_per_s": 1e3 / ms, "ms_per_grad": ms,
            "steps": w["steps"], "cells": nx * ny * nz, "ckpt_outer_inner": [k_outer, k_inner],
            "device_gb": dev_bytes / 1e9, "forward_steps": fwd_steps, "loss": loss,
            "grad_pos": [float(v) for v in gpos], "grad_signal_norm": float(np.linalg.norm(gsig)),
            "launches": launches, "fwd_equiv_glups": nx * ny * nz * w["steps"] / (ms / 1e3) / 1e9}


def family_a_cpu(name, seconds=5.0):
    """The unmodified family-A reference program (01, 02, 03 or 04 through
    oracle/_ref, FP64, OpenMP on all host threads) on its own domain (01, 04)
    or a sub-domain of its own set-up (02, 03), in GLUPS; None where the
    harness was not built."""
    import oracle

    which = {"scattering_a": "01", "lloyd_a": "02", "doppler_a": "03", "hpc_a": "04"}[name]
    if not oracle.refa_available(which):
        return None
    if which == "01":
        p = dict(x_min=-8.0, x_max=8.0, y_min=-8.0, y_max=8.0, z_min=-0.2, z_max=0.2, dx=0.05, amp=0.01)
    elif which == "04":
        p = dict(x_min=-13.0, x_max=13.0, y_min=-13.0, y_max=13.0, z_min=-13.0, z_max=13.0, dx=0.125, amp=0.01)
    elif which == "02":
        p = dict(x_min=-10.0, x_max=10.0, y_min=-10.0, y_max=10.0, z_min=-2.0, z_max=10.0, dx=0.2, amp=0.5,
                 b_param=2.0)
    else:
        p = dict(x_min=0.0, x_max=25.0, y_min=0.0, y_max=25.0, z_min=0.0, z_max=37.5, dx=0.25, amp=0.01, Ma=0.2,
                 tau_bulk=0.51, tau_sponge_max=0.9, sponge_width=20)
    ref = oracle.RefASolver(which, **p)
    nx, ny, nz = (d - 2 for d in ref.dims_halo)
    ref.step(1)
    n, t = 0, 0.0
    while t < seconds:
        t0 = time.perf_counter()
        ref.step(2)
        t += time.perf_counter() - t0
        n += 2
    return {"value": nx * ny * nz * n / t / 1e9, "unit": "GLUPS", "cores": os.cpu_count(), "kind": "reference",
            "sample": f"{nx}x{ny}x{nz} {'domain' if which in ('01', '04') else 'sub-domain'}, {n} steps of "
                      "exchange_halos+step, FP64"}


# The reference arm's sample: a 256x256 plan window of the headline city (the
# 2048x2048x256 generator, seed 2024), 128 layers.  An FP64 run of the whole
# headline grid would need about 330 GB of host memory (19 x 8 B x 2 buffers
# per cell), so the reference is timed on this window as a rate.
REF_WINDOW = (896, 896, 256, 128)   # x0, y0, width, layers


def reference_sample():
    """Triangles of the window, built by the pure-Python restatement of the
    city generator (oracle/city.py), so the reference arm maps no library of
    the product."""
    from oracle import city

    x0, y0, w, _ = REF_WINDOW
    boxes, _ = city.city_boxes(2048, 2048, 2024, fp=(20, 60), height=(10, 80), coverage=0.40, street=8, margin=40)
    part = city.crop_boxes(boxes, x0, y0, x0 + w, y0 + w)
    tris = np.concatenate([city.box_triangles(*b) for b in part]) if part else np.zeros((0, 9), np.float32)
    return tris


def cpu_baseline(steps_hint=None, seconds=12.0):
    """The reference's CPU step on the bounded sample (rank 0, N=1): the
    unmodified 06 (oracle/_ref/libref06.so: apply_source, exchange_halos,
    step_collision_bgk, FP64, OpenMP on every host thread), or the FP64 port
    where the reference was not built."""
    import oracle
    from oracle import city

    _, _, w, nz = REF_WINDOW
    nx = ny = w
    tris = reference_sample()
    threads = os.cpu_count() or 1
    if oracle.ref_available("06"):
        stl = "/tmp/bench_city_window.stl"
        city.stl_write(stl, tris)
        ref = oracle.RefSolver("06", (0, nx), (0, ny), (0, nz), 1.0, 0.51, (128.5, 128.5, 2.5, 128.5, 128.5, 2.5,
                                                                           0.0, 10.0, 0.0), stl=stl)
        kind = "reference"

        def run(n):
            ref.step(n)
    else:
        from nlos_lbm import abi
        cfg = abi.reference_config(x_min=0.0, x_max=float(nx), y_min=0.0, y_max=float(ny), z_min=0.0,
                                   z_max=float(nz), dx=1.0, c_phys=abi.CS, tau=0.51)
        src = abi.reference_source(sx=128.5, sy=128.5, sz=2.5, ex=128.5, ey=128.5, ez=2.5, amp=1e-3, t0=40.0,
                                   sigma_t=8.0)
        orc = oracle.OracleSolver(cfg, [src], None, triangles=tris)
        kind = "port"

        def run(n):
            orc.step(n)
    run(1)   # warm-up
    t0 = time.perf_counter()
    run(2)
    per = (time.perf_counter() - t0) / 2
    n = steps_hint or max(2, min(200, int(seconds / max(per, 1e-6))))
    t0 = time.perf_counter()
    run(n)
    dt = time.perf_counter() - t0
    cells = nx * ny * nz
    x0, y0 = REF_WINDOW[:2]
    return dict(value=cells * n / dt / 1e9, unit=UNIT, cores=threads, kind=kind,
                sample=f"{nx}x{ny}x{nz} window [{x0},{x0 + nx})x[{y0},{y0 + ny}) of the 2048x2048x256 city (an FP64 "
                       f"run of the whole grid needs ~330 GB of host memory), timed as a rate: {n} full steps "
                       f"(apply_source+exchange_halos+step_collision_bgk), FP64, {threads} threads",
                seconds=dt, steps=n)


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle

    oracle_kind = "reference" if oracle.ref_available("06") else "port"
    # each timed step of the sample is one reference step; the whole run is bounded
    b = cpu_baseline(steps_hint=max(1, args.steps))
    line = {"metric": METRIC, "value": b["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": b["steps"],
            "warmup": args.warmup, "ms_per_step": b["seconds"] / b["steps"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "impl": "reference",
            "config": headline_config(args.workload, args.storage, args.gpus),
            "cpu_baseline": {"value": b["value"], "unit": UNIT, "cores": b["cores"], "kind": oracle_kind,
                             "sample": b["sample"]},
            "e2e": {"value": b["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_slab_arm(args, torch, dist, world, rank, local, barrier, reduce_max):
    """Strong scaling: one z-slab of the headline grid per rank, the cut
    messages (crossing populations only) moved by NCCL point-to-point."""
    import nlos_lbm
    from nlos_lbm import ranks, workloads

    hbm_peak, peak_kind = measured_peaks()
    storage = None if args.storage is None else (1 if args.storage == "fp16" else 0)
    w = workloads.build(args.workload, storage=storage)
    r = ranks.SlabRank(w["cfg"], dist, w["sources"], w["probes"], triangles=w["triangles"], device=local,
                       staging="device")
    nx, ny, nz = workloads.cells(w["cfg"])
    cells = nx * ny * nz
    r.step(args.warmup)
    stream = r.stream
    l0 = r.solver.launch_count
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        r.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
    ms = reduce_max(e0.elapsed_time(e1))
    launches = r.solver.launch_count - l0
    h0, d0 = r.solver.transfer_bytes()
    t0 = time.perf_counter()
    r.step(args.steps)
    r.solver.get_probes()
    e2e_ms = reduce_max((time.perf_counter() - t0) * 1e3)
    h1, d1 = r.solver.transfer_bytes()
    clocks = clk.summary()
    value = cells * args.steps / (ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "fp16-store/fp32-compute" if w["cfg"].storage == 1 else "fp32",
            "data": DATA,
            "config": {"workload": f"{args.workload}: {w['description']}", "grid": [nx, ny, nz],
                       "parallelism": f"z-slabs x{world}", "slab_bounds": r.bounds,
                       "message_bytes_per_cut": r.lib.lbm_slab_message_bytes(r.h)},
            "e2e": {"value": cells * args.steps / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": (h1 - h0) / args.steps, "d2h_bytes_per_step": (d1 - d0) / args.steps},
            "gpu_launches": launches, "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "roofline": {"bound": "hbm", "peak": hbm_peak, "unit": "GB/s", "peak_kind": peak_kind,
                         "achieved": cells / world * (76 if w["cfg"].storage == 1 else 152) / (ms / args.steps / 1e3) / 1e9,
                         "traffic": None}}
    line["roofline"]["frac"] = line["roofline"]["achieved"] / hbm_peak
    if rank == 0:
        print(json.dumps(line), flush=True)
    r.close()
    return 0


def run_our_arm(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    barrier, reduce_max = make_reducers(dist, "cuda")
    if args.split == "slab":
        rc = run_slab_arm(args, torch, dist, world, rank, local, barrier, reduce_max)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return rc

    hbm_peak, peak_kind = measured_peaks()
    headline = args.workload
    with ClockSampler(local) as clk:
        storage = None if args.storage is None else (1 if args.storage == "fp16" else 0)
        s, w, head = measure(headline, storage, args.steps, args.warmup, local, torch, barrier, reduce_max)
    clocks = clk.summary()
    # e2e through the C-ABI with host buffers (same workload, same handle)
    e2e_ms, h2d_ps, d2h_ps = e2e_measure(s, w, args.steps)
    e2e_ms = reduce_max(e2e_ms)
    del s
    import gc

    gc.collect()

    secondary = {}
    series = {}
    if world == 1 and not args.headline_only:
        for nm, st in (("city1024", 0), ("city1024", 1)):
            s2, _, r = measure(nm, st, args.steps, args.warmup, local, torch, barrier, reduce_max)
            secondary[f"{nm}_{r['storage']}"] = {k: r[k] for k in ("glups_rank", "ms", "kernel_ms_avg", "dims",
                                                                    "bytes_per_cell", "fluid_fraction")}
            secondary[f"{nm}_{r['storage']}"]["hbm_frac_kernel"] = (
                r["cells"] * r["bytes_per_cell"] / (r["kernel_ms_avg"] / 1e3) / 1e9 / hbm_peak)
            # the probe error of the metric: both storages run on to the same
            # step, then the FP16 series is compared with the FP32 one (FP32 is
            # within a few 1e-6 of the FP64 oracle in the parity tests)
            s2.step(max(0, ERR_STEPS - s2.step_count))
            series[r["storage"]] = s2.get_probes()[:ERR_STEPS]
            del s2
            gc.collect()
        a, b = series["fp16"], series["fp32"]
        secondary["fp16_probe_rel_l2_vs_fp32"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
        secondary["fp16_probe_error_steps"] = ERR_STEPS

    family_a = {}
    if world == 1 and not args.headline_only:
        # the reference's family-A programs at their own sizes on scheme A (FP32)
        for nm in ("lloyd_a", "doppler_a", "scattering_a", "hpc_a"):
            s2, _, r = measure(nm, None, args.steps, args.warmup, local, torch, barrier, reduce_max)
            family_a[nm] = {k: r[k] for k in ("glups_rank", "ms", "kernel_ms_avg", "dims", "bytes_per_cell",
                                               "description", "fluid_fraction")}
            family_a[nm]["hbm_frac_kernel"] = (r["cells"] * r["bytes_per_cell"] / (r["kernel_ms_avg"] / 1e3) / 1e9
                                               / hbm_peak)
            if nm == "hpc_a":
                # 04's own benchmark: 2000 steps after 100 (04:360-404), its MLUPS over all cells
                from nlos_lbm import workloads

                s2.step(max(0, 100 - s2.step_count))
                w2 = workloads.build(nm)
                ms2 = device_timed_steps(s2, w2["steps"], torch, barrier)
                family_a[nm]["program_steps"] = w2["steps"]
                family_a[nm]["program_ms"] = ms2
                family_a[nm]["mlups"] = r["cells"] * w2["steps"] / (ms2 / 1e3) / 1e6
            if not args.no_cpu:
                family_a[nm]["cpu_reference"] = family_a_cpu(nm)
            del s2
            gc.collect()

    adjoint = None
    if world == 1 and not args.headline_only and not args.no_adjoint:
        adjoint = adjoint_measure(local, torch)
        gc.collect()

    n = world
    cells, steps = head["cells"], head["steps"]
    value = replica_glups(n, cells, steps, head["ms"])
    achieved = cells * head["bytes_per_cell"] / (head["kernel_ms_avg"] / 1e3) / 1e9
    # DRAM bytes per cell update measured by ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum) on one launch of the fused step on the
    # 512x512x128 city; traffic grows with the cell count, so one launch here
    # moves cells times that.
    per_cell = NCU_TRAFFIC_PER_CELL.get(head["storage"])
    traffic = None if per_cell is None else per_cell * cells
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "k_step_hw" if head["storage"] == "fp16" else "k_step",
                "kernel_ms": head["kernel_ms_avg"], "bytes_per_cell": head["bytes_per_cell"]}
    for key in ("city1024_fp32", "city1024_fp16"):
        if key in secondary:
            roofline[key + "_frac"] = secondary[key]["hbm_frac_kernel"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": steps, "warmup": args.warmup,
        "ms_per_step": head["ms"] / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp16-store/fp32-compute" if head["storage"] == "fp16" else "fp32",
        "data": DATA,
        "config": headline_config(headline, head["storage"], n, head["dims"], head["description"]),
        "roofline": roofline,
        "e2e": {"value": n * cells * steps / (e2e_ms / 1e3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d_ps,
                "d2h_bytes_per_step": d2h_ps},
        "gpu_launches": head["launches"],
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "fluid_glups": value * head["fluid_fraction"],
    }
    if secondary.get("city1024_fp32") and secondary.get("city1024_fp16"):
        line["fp16_over_fp32"] = secondary["city1024_fp16"]["glups_rank"] / secondary["city1024_fp32"]["glups_rank"]
        line["fp16_probe_rel_l2"] = secondary["fp16_probe_rel_l2_vs_fp32"]
    if adjoint is not None:
        line["adjoint_grad_per_s"] = adjoint["grad_per_s"]
    if world == 1 and rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline().items() if k in ("value", "unit", "cores", "kind",
                                                                                  "sample")}
    if rank == 0:
        # the legs first, one JSON object per line; the headline line last
        if secondary:
            print(json.dumps({"leg": "city1024 FP32 and FP16 storage, FP16 probe error against FP32",
                              **secondary}), flush=True)
        for nm, v in family_a.items():
            print(json.dumps({"leg": "family_a " + nm, **v}), flush=True)
        if adjoint is not None:
            print(json.dumps({"leg": "adjoint", **adjoint}), flush=True)
        print(json.dumps({"leg": "headline details", "probes_finite": head["probes_finite"],
                          "fluid_fraction": head["fluid_fraction"], "plan_coverage": head["coverage"],
                          "f16_scale": head["f16_scale"], "clock_samples": clocks.get("samples")}), flush=True)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="city2048",
                    choices=["city2048", "city1024", "city512", "lloyd", "scatter", "lloyd_a", "lloyd_a_small",
                             "doppler_a", "scattering_a", "hpc_a"])
    ap.add_argument("--storage", default=None, choices=["fp32", "fp16"],
                    help="population storage of the headline workload (default: the workload's own)")
    ap.add_argument("--split", default="replicas", choices=["replicas", "slab"],
                    help="multi-GPU form: independent replicas (weak scaling, the default) or one z-slab of the "
                         "headline grid per rank (strong scaling)")
    ap.add_argument("--headline-only", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="time lbm_adjoint_grad alone and print its JSON object (profiling runs)")
    ap.add_argument("--adjoint-workload", default="adjoint256", choices=["adjoint256", "adjoint128"])
    ap.add_argument("--adjoint-steps", type=int, default=None, help="override the adjoint run length")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.adjoint_only:
        import torch

        torch.cuda.set_device(0)
        print(json.dumps(adjoint_measure(0, torch, workload=args.adjoint_workload, steps=args.adjoint_steps)),
              flush=True)
        return 0
    return run_our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
