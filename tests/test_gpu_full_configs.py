"""Parity at the configured sizes and lengths of the benchmark workloads.

* The localisation gradient on the 256x256x128 patch over its 3000 steps
  (64 receivers, 200-step checkpoints, the schedule the bench runs: most
  of the run's moments kept from the first pass) against central differences
  of the GPU's own FP32 forward at h = 1e-2 cells, and its signal gradient
  against one directional difference.  Bound: 1e-4 relative (the gradient
  accuracy target of the localisation benchmark).  A second call gives the
  same bits.
* The checkpoint schedule with recomputed segments AND a stored tail, at an
  intermediate size (112x96x48, 600 steps, 200-step checkpoints, memory
  capped with NLOS_LBM_ADJ_BUDGET) against the FP64 CPU discrete adjoint of
  the oracle: 1e-4 relative, and bit-identical to the all-recompute schedule.
* The FP16 and FP32 storages on the 1024x1024x256 city over its whole 4000
  steps: the FP16 probe series within 1e-3 relative L2 of the FP32 one (FP32
  is held to the FP64 oracle at 1e-5 on the 256x256x128 patch of the same
  physics over 4000 steps, test_gpu_parity.py).

The forward these gradients differentiate is the reference's family-B step
(06_transient_localization_dx1.cpp:906-972) with its probe record
(06:1085-1092); the reference itself has no adjoint.
"""
import numpy as np
import pytest

import scenarios
from nlos_lbm import Solver, abi, workloads
from oracle import OracleSolver
from scenarios import rel_l2
from test_gpu_adjoint import _partial_tail_budget

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
FP16_PROBE_TOL = 1e-3
H = 1e-2   # cells (dx = 1)


def _loss(w, src, observed, steps):
    g = Solver(w["cfg"], [src], w["probes"], triangles=w["triangles"])
    g.step(steps)
    p = g.get_probes()
    g.close()
    return scenarios.misfit(p, observed)


def test_full_size_gradient_matches_central_differences(gpu):
    w = workloads.build("adjoint256")
    steps = w["steps"]
    truth = Solver(w["cfg"], [w["true_source"]], w["probes"], triangles=w["triangles"])
    truth.step(steps)
    observed = truth.get_probes()
    truth.close()
    trial = w["sources"][0]
    g = Solver(w["cfg"], [trial], w["probes"], triangles=w["triangles"])
    k_outer, k_inner, _, fwd = g.adjoint_plan(steps, 200, 0)
    # the schedule the bench runs: the first pass keeps the moments of as many 200-step segments
    # as fit (most of the run at 6 bytes per cell), the rest are recomputed once
    assert k_outer == 200 and steps <= fwd < 2 * steps - 1
    L, gp, gs, pred = g.adjoint_grad(observed, 200, 0)
    # the small kernels that run on the second stream beside the steps leave no trace:
    # a second call gives the same bits
    again = g.adjoint_grad(observed, 200, 0)
    g.close()
    assert again[0] == L
    for a, b in zip(again[1:], (gp, gs, pred)):
        assert np.array_equal(a, b)
    assert L == pytest.approx(_loss(w, trial, observed, steps), rel=1e-12)
    assert np.max(np.abs(gp)) > 0
    fd = []
    for a in range(3):
        lp = _loss(w, scenarios.source_copy(trial, H * np.eye(3)[a])[0], observed, steps)
        lm = _loss(w, scenarios.source_copy(trial, -H * np.eye(3)[a])[0], observed, steps)
        fd.append((lp - lm) / (2 * H))
    fd = np.array(fd)
    assert np.max(np.abs(fd - gp)) <= GRAD_TOL * np.max(np.abs(gp)), (fd, gp)
    # the signal: the misfit is quadratic in it, so one large symmetric step is exact
    sig = scenarios.source_signal(trial, steps, 1.0)
    v = np.random.default_rng(3).standard_normal(steps)
    eps = 0.05 * np.max(np.abs(sig))
    srcp, keep_p = scenarios.source_copy(trial, table=sig + eps * v)
    srcm, keep_m = scenarios.source_copy(trial, table=sig - eps * v)
    fdv = (_loss(w, srcp, observed, steps) - _loss(w, srcm, observed, steps)) / (2 * eps)
    del keep_p, keep_m
    assert fdv == pytest.approx(float(gs @ v), rel=GRAD_TOL)


def test_stored_tail_and_recompute_schedule_matches_fp64_adjoint(gpu, monkeypatch):
    sc = scenarios.adjoint_scenario(nx=112, ny=96, nz=48, steps=600, nprobe=24, seed=5)
    steps = sc["steps"]
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    # a cap under which the first segments are recomputed and the rest kept from the first pass
    budget, plan, none = _partial_tail_budget(g, steps, 200, monkeypatch)
    assert plan[:2] == (200, 200)
    monkeypatch.setenv("NLOS_LBM_ADJ_BUDGET", str(budget))
    part = g.adjoint_grad(sc["observed"], 200, 0)
    monkeypatch.delenv("NLOS_LBM_ADJ_BUDGET")
    rec = g.adjoint_grad(sc["observed"], 200, 200)
    assert part[0] == rec[0]
    for a, b in zip(part[1:], rec[1:]):
        assert np.array_equal(a, b)
    L, gp, gs, pred = part
    o = OracleSolver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    L0, gp0, gs0, pred0 = o.adjoint_grad(sc["observed"], K=25)
    assert rel_l2(pred, pred0) <= 1e-5, rel_l2(pred, pred0)
    assert L == pytest.approx(L0, rel=GRAD_TOL)
    assert np.max(np.abs(gp - gp0)) <= GRAD_TOL * np.max(np.abs(gp0)), (gp, gp0)
    assert rel_l2(gs, gs0) <= GRAD_TOL, rel_l2(gs, gs0)


def test_fp16_city1024_over_its_full_length_matches_fp32(gpu):
    series = {}
    for storage in (abi.LBM_STORE_F32, abi.LBM_STORE_F16):
        w = workloads.build("city1024", storage=storage)
        g = Solver(w["cfg"], w["sources"], w["probes"], triangles=w["triangles"])
        g.step(w["steps"])
        series[storage] = g.get_probes()
        g.close()
    a, b = series[abi.LBM_STORE_F16], series[abi.LBM_STORE_F32]
    assert a.shape == b.shape == (4000, 256)
    assert np.all(np.isfinite(a)) and np.max(np.abs(b)) > 0
    assert rel_l2(a, b) <= FP16_PROBE_TOL, rel_l2(a, b)
