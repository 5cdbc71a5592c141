"""The FP64 CPU discrete adjoint of the oracle (the checker of the GPU
adjoint) against central finite differences of the oracle's own FP64
forward, on a small synthetic-city patch.  No GPU.

Tolerances: with trilinear injection and all eight injection cells FLUID the
probe series is linear in a shift of the source, so the misfit is quadratic
and the central difference is exact up to rounding (measured 5e-10); the
Gaussian stencil has an O(h^2) truncation error (measured 3e-5 at h = 1e-2
cells).  The misfit is quadratic in the source signal, so the directional
difference is exact up to rounding.
"""
import numpy as np
import pytest

import scenarios
from nlos_lbm import abi
from oracle import OracleSolver

H = 1e-2   # cells (dx = 1)


def _loss(sc, shift=(0.0, 0.0, 0.0), table=None):
    src, keep = scenarios.source_copy(sc["trial"], shift, table)
    o = OracleSolver(sc["cfg"], [src], sc["probes"], triangles=sc["triangles"])
    o.step(sc["steps"])
    del keep
    return scenarios.misfit(o.get_probes(), sc["observed"])


@pytest.fixture(scope="module", params=[abi.LBM_INJECT_TRILINEAR, abi.LBM_INJECT_GAUSS], ids=["trilinear", "gauss"])
def case(request):
    sc = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=80, nprobe=8, injection=request.param)
    o = OracleSolver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    return sc, o.adjoint_grad(sc["observed"], K=9)


def test_fp64_adjoint_position_matches_central_fd(case):
    sc, (L, gpos, _, pred) = case
    assert L == pytest.approx(scenarios.misfit(pred, sc["observed"]), rel=1e-14)
    assert L == pytest.approx(_loss(sc), rel=1e-13)
    fd = np.array([(_loss(sc, H * np.eye(3)[a]) - _loss(sc, -H * np.eye(3)[a])) / (2 * H) for a in range(3)])
    tol = 1e-7 if sc["trial"].injection == abi.LBM_INJECT_TRILINEAR else 1e-4
    assert np.max(np.abs(fd - gpos)) <= tol * np.max(np.abs(gpos)), (fd, gpos)


def test_fp64_adjoint_signal_matches_directional_fd(case):
    sc, (L, _, gsig, _) = case
    o = OracleSolver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    sig = scenarios.source_signal(sc["trial"], sc["steps"], o.dt)
    assert _loss(sc, table=sig) == pytest.approx(L, rel=1e-12)   # the table reproduces the Ricker run
    v = np.random.default_rng(0).standard_normal(sc["steps"])
    eps = 1e-3 * np.max(np.abs(sig))
    fd = (_loss(sc, table=sig + eps * v) - _loss(sc, table=sig - eps * v)) / (2 * eps)
    assert fd == pytest.approx(float(gsig @ v), rel=1e-7)


def test_fp64_adjoint_is_independent_of_checkpoint_interval():
    sc = scenarios.adjoint_scenario(nx=24, ny=20, nz=12, steps=30, nprobe=4)
    res = []
    for K in (1, 4, 30):
        o = OracleSolver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
        res.append(o.adjoint_grad(sc["observed"], K=K))
    for r in res[1:]:
        assert r[0] == res[0][0]
        assert np.array_equal(r[1], res[0][1])
        assert np.array_equal(r[2], res[0][2])
