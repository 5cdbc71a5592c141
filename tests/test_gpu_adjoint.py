"""Reverse-time adjoint on the GPU (lbm_adjoint_grad) against the FP64 CPU
discrete adjoint of the oracle and against central finite differences of the
GPU's own FP32 forward, on synthetic-city patches.

Tolerances, stated per check:
  - vs the FP64 adjoint: 1e-4 relative (the gradient accuracy target of the
    localisation benchmark), on the position gradient (max-norm) and on the
    per-step signal gradient (relative L2); the forward series within the FP32
    probe bar 1e-5;
  - vs central differences of the FP32 forward at h = 1e-2 cells: 1e-4
    relative on the position gradient;
  - checkpoint schedules: bit-identical gradients (the recomputation is
    deterministic and no probe shares a cell with another).
"""
import numpy as np
import pytest

import scenarios
from nlos_lbm import LBMError, Solver, abi
from oracle import OracleSolver
from scenarios import rel_l2

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
PROBE_TOL = 1e-5
H = 1e-2   # cells (dx = 1)


def _gpu_loss(sc, shift=(0.0, 0.0, 0.0), table=None):
    src, keep = scenarios.source_copy(sc["trial"], shift, table)
    g = Solver(sc["cfg"], [src], sc["probes"], triangles=sc["triangles"])
    g.step(sc["steps"])
    p = g.get_probes()
    g.close()
    del keep
    return scenarios.misfit(p, sc["observed"])


CASES = {
    "trilinear": dict(injection=abi.LBM_INJECT_TRILINEAR),
    "gauss": dict(injection=abi.LBM_INJECT_GAUSS),
    "moving": dict(injection=abi.LBM_INJECT_TRILINEAR, speed=0.05),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    sc = scenarios.adjoint_scenario(**CASES[request.param])
    o = OracleSolver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    ref = o.adjoint_grad(sc["observed"], K=16)
    return request.param, sc, ref


def test_adjoint_matches_fp64_adjoint(case, gpu):
    name, sc, (L0, gp0, gs0, pred0) = case
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    L, gp, gs, pred = g.adjoint_grad(sc["observed"], ckpt_outer=50, ckpt_inner=8)
    assert rel_l2(pred, pred0) <= PROBE_TOL, rel_l2(pred, pred0)
    assert L == pytest.approx(L0, rel=GRAD_TOL)
    assert np.max(np.abs(gp - gp0)) <= GRAD_TOL * np.max(np.abs(gp0)), (gp, gp0)
    assert rel_l2(gs, gs0) <= GRAD_TOL, rel_l2(gs, gs0)


def test_adjoint_matches_central_fd_of_gpu_forward(case, gpu):
    """Every case: the trilinear misfit is piecewise quadratic in the shift
    (exact central differences inside a cell), the Gaussian stencil's adds an
    O(h^2) term (3e-5 relative at h = 1e-2 in the FP64 oracle's own check);
    both sit inside the 1e-4 bar."""
    name, sc, _ = case
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    L, gp, gs, _ = g.adjoint_grad(sc["observed"])
    g.close()
    assert L == pytest.approx(_gpu_loss(sc), rel=1e-12)   # same forward, same FP64 misfit
    fd = np.array([(_gpu_loss(sc, H * np.eye(3)[a]) - _gpu_loss(sc, -H * np.eye(3)[a])) / (2 * H)
                   for a in range(3)])
    assert np.max(np.abs(fd - gp)) <= GRAD_TOL * np.max(np.abs(gp)), (fd, gp)
    # signal: the misfit is quadratic in the signal, so a large step is exact
    sig = scenarios.source_signal(sc["trial"], sc["steps"], 1.0)
    v = np.random.default_rng(1).standard_normal(sc["steps"])
    eps = 0.05 * np.max(np.abs(sig))
    fdv = (_gpu_loss(sc, table=sig + eps * v) - _gpu_loss(sc, table=sig - eps * v)) / (2 * eps)
    assert fdv == pytest.approx(float(gs @ v), rel=GRAD_TOL)


def test_checkpoint_schedules_are_bit_identical(gpu):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=45, nprobe=6)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    # (0, 0) and (10, 0): the whole run's forward data kept from the first pass
    runs = [g.adjoint_grad(sc["observed"], a, b) for a, b in ((0, 0), (45, 45), (7, 3), (1, 1), (10, 10), (10, 0))]
    for r in runs[1:]:
        assert r[0] == runs[0][0]
        assert np.array_equal(r[1], runs[0][1])
        assert np.array_equal(r[2], runs[0][2])
        assert np.array_equal(r[3], runs[0][3])


def test_adjoint_returns_to_rest_state(gpu):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=40, nprobe=6)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    g.step(17)                                   # any prior state is discarded
    _, _, _, pred = g.adjoint_grad(sc["observed"], 9, 4)
    assert g.step_count == 0
    assert g.get_probes().shape[0] == 0
    g.step(sc["steps"])
    assert np.array_equal(g.get_probes(), pred)  # the forward of the adjoint is lbm_step's


def test_nan_observations_and_outside_probes_are_skipped(gpu):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=40, nprobe=6)
    probes = np.vstack([sc["probes"], [[-5.0, 3.0, 3.0]]])        # last probe outside the grid
    obs = np.hstack([sc["observed"], np.zeros((sc["steps"], 1))])
    obs[:, 0] = np.nan                                            # probe 0 unobserved
    g = Solver(sc["cfg"], [sc["trial"]], probes, triangles=sc["triangles"])
    L, gp, gs, pred = g.adjoint_grad(obs)
    assert np.all(np.isnan(pred[:, -1]))
    ref = Solver(sc["cfg"], [sc["trial"]], sc["probes"][1:], triangles=sc["triangles"])
    L1, gp1, gs1, _ = ref.adjoint_grad(sc["observed"][:, 1:])
    assert L == L1
    assert np.array_equal(gp, gp1) and np.array_equal(gs, gs1)


def test_adjoint_rejects_unsupported_set_ups(gpu):
    sc = scenarios.adjoint_scenario(nx=24, ny=20, nz=12, steps=10, nprobe=3)
    f16 = scenarios.lattice_config(24, 20, 12, 0.52, storage=abi.LBM_STORE_F16, f16_scale=1e3)
    g = Solver(f16, [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    with pytest.raises(LBMError) as e:
        g.adjoint_grad(sc["observed"])
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
    g = Solver(sc["cfg"], [sc["trial"], sc["true"]], sc["probes"], triangles=sc["triangles"])
    with pytest.raises(LBMError) as e:
        g.adjoint_grad(sc["observed"])
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
    g = Solver(sc["cfg"], [sc["trial"]], None, triangles=sc["triangles"])
    with pytest.raises(LBMError) as e:
        g.adjoint_grad(np.zeros((10, 0)))
    assert e.value.status == abi.LBM_ERR_STATE


def test_adjoint_plan(gpu):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=45, nprobe=6)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    assert g.adjoint_plan(45, 7, 3)[:2] == (7, 3)
    assert g.adjoint_plan(45, 100, 60)[:2] == (45, 45)            # intervals clamp to the run
    o, i, nbytes, fwd = g.adjoint_plan(45, 0, 0)                   # small grid: the whole run's forward
    assert (o, i) == (45, 45) and nbytes > 0 and fwd == 45          # data fits, no recompute
    o, i, nbytes, fwd = g.adjoint_plan(45, 10, 0)
    assert (o, i) == (10, 10) and fwd == 45
    assert g.adjoint_plan(45, 45, 45)[3] == 2 * 45 - 1              # one forward pass + one recompute
    assert g.adjoint_plan(45, 9, 1)[3] > g.adjoint_plan(45, 9, 9)[3]


def _partial_tail_budget(g, steps, outer, monkeypatch):
    """A memory cap under which the plan keeps the forward data of some but
    not all segments (some recomputed, a stored tail): searched between the
    all-recompute plan's bytes and the uncapped plan's."""
    none = g.adjoint_plan(steps, outer, outer)        # explicit inner interval: every segment recomputed
    full = g.adjoint_plan(steps, outer, 0)            # small grid: the whole run's forward data fits
    assert full[3] == steps and none[3] > steps
    assert full[2] > none[2], "storing every step must cost more than the checkpoints for a partial tail"
    for f in np.linspace(0.05, 0.95, 19):
        budget = none[2] + f * (full[2] - none[2])
        monkeypatch.setenv("NLOS_LBM_ADJ_BUDGET", str(budget))
        plan = g.adjoint_plan(steps, outer, 0)
        monkeypatch.delenv("NLOS_LBM_ADJ_BUDGET")
        if steps < plan[3] < none[3]:
            return budget, plan, none
    raise AssertionError("no cap between the two plans gives a partial tail")


def test_partial_stored_tail(gpu, monkeypatch):
    """A memory cap that holds the forward data of the last segments only:
    those are reversed from the first pass's data, the others with a
    recompute; the result is bit-identical to recomputing every segment."""
    # 120 steps in 20-step segments: keeping every step's forward data needs more memory than the
    # full-state checkpoints of an all-recompute plan, so caps in between give a partial tail
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=120, nprobe=6)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    budget, plan, none = _partial_tail_budget(g, 120, 20, monkeypatch)
    assert plan[:2] == (20, 20)
    monkeypatch.setenv("NLOS_LBM_ADJ_BUDGET", str(budget))
    part = g.adjoint_grad(sc["observed"], 20, 0)
    monkeypatch.delenv("NLOS_LBM_ADJ_BUDGET")
    ref = g.adjoint_grad(sc["observed"], 20, 20)
    assert part[0] == ref[0]
    for a, b in zip(part[1:], ref[1:]):
        assert np.array_equal(a, b)


def test_workspace_is_kept_and_released(gpu):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=40, nprobe=6)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    r1 = g.adjoint_grad(sc["observed"], 9, 4)
    r2 = g.adjoint_grad(sc["observed"][:20], 9, 4)    # smaller run in the kept workspace
    r3 = g.adjoint_grad(sc["observed"], 9, 4)
    g.adjoint_release()
    r4 = g.adjoint_grad(sc["observed"], 9, 4)         # fresh workspace
    for r in (r3, r4):
        assert r[0] == r1[0] and np.array_equal(r[1], r1[1]) and np.array_equal(r[2], r1[2])
    assert r2[2].shape == (20,)
