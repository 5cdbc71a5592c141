"""The L2 prefetches of the latency-bound kernels are hints only: the
adjoint step's (NLOS_LBM_ADJ_PREFETCH_ROWS) and the scheme-A instance with
per-column fields (04's, NLOS_LBM_A_PREFETCH_ROWS) give the same bits with
the prefetch off, at the default distance and at a distance past the end
of the grid, on grids whose rows are not whole multiples of a CTA's
columns.  Each prefetch is one cp.async.bulk.prefetch.L2 of a contiguous,
16-byte aligned range inside the buffer it hints at."""
import numpy as np
import pytest

import scenarios
from nlos_lbm import Solver

pytestmark = pytest.mark.gpu


def _column_run(sc, monkeypatch, rows):
    if rows is None:
        monkeypatch.delenv("NLOS_LBM_A_PREFETCH_ROWS", raising=False)
    else:
        monkeypatch.setenv("NLOS_LBM_A_PREFETCH_ROWS", str(rows))
    g = Solver(sc["cfg"], sc["sources"], sc["probes"], mask=sc["mask"], blend_xy=sc.get("blend_xy"),
               field_xy=sc.get("field_xy"))
    g.step(sc["steps"])
    out = g.get_probes(), g.get_rho()
    g.close()
    return out


@pytest.mark.parametrize("n", [40, 45])
def test_column_instance_prefetch_changes_no_bit(n, monkeypatch, gpu):
    sc = scenarios.family_a("hpc_a", n=n, steps=24)
    ref = _column_run(sc, monkeypatch, 0)
    assert np.max(np.abs(ref[0])) > 0
    for rows in (None, 1, 100000):
        got = _column_run(sc, monkeypatch, rows)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), rows


@pytest.mark.parametrize("dims", [(48, 40, 24), (67, 30, 21)])
def test_adjoint_prefetch_changes_no_bit(dims, monkeypatch, gpu):
    nx, ny, nz = dims
    sc = scenarios.adjoint_scenario(nx=nx, ny=ny, nz=nz, steps=60, nprobe=8, seed=3)
    g = Solver(sc["cfg"], [sc["trial"]], sc["probes"], triangles=sc["triangles"])
    monkeypatch.setenv("NLOS_LBM_ADJ_PREFETCH_ROWS", "0")
    ref = g.adjoint_grad(sc["observed"], 20, 0)
    assert np.max(np.abs(ref[1])) > 0
    for rows in (None, 7, 100000):
        if rows is None:
            monkeypatch.delenv("NLOS_LBM_ADJ_PREFETCH_ROWS")
        else:
            monkeypatch.setenv("NLOS_LBM_ADJ_PREFETCH_ROWS", str(rows))
        got = g.adjoint_grad(sc["observed"], 20, 0)
        assert got[0] == ref[0], rows
        for a, b in zip(got[1:], ref[1:]):
            assert np.array_equal(a, b), rows
    g.close()
