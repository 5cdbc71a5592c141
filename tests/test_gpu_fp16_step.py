"""The fused FP16 step (warp pipelines of cp.async copies into shared
memory) against the FP64 oracle.  The cases cover one partial block per row
(nx < 64), exactly one block, several blocks with a partial last one, open x
faces (NSCBC ghosts at both row ends), buildings (links and bounce-back) and
more rows than resident warps.
"""
import numpy as np
import pytest

import nlos_lbm
import oracle
import scenarios
from nlos_lbm import abi
from scenarios import rel_l2

pytestmark = pytest.mark.gpu

# FP16 deviation storage with scale 1/amplitude: the 1e-3 probe target
FP16_PROBE_TOL = 1e-3


def wide_box(nx=200, ny=24, nz=20, steps=100):
    """Open box (NSCBC on every face) four blocks wide with a partial last
    block, a rigid box crossing a block boundary, a Gaussian pulse; the
    probes sit where the pulse is well above the FP16 resolution."""
    cfg = scenarios.lattice_config(nx, ny, nz, 0.55, face_bc=(abi.LBM_BC_NSCBC,) * 6, sponge_faces=(1 << 6) - 1,
                                   sponge_width=6.0, sponge_strength=0.5, storage=abi.LBM_STORE_F16,
                                   f16_scale=1000.0)
    tris = scenarios.boxes_to_triangles([(56, 6, 5, 74, 16, 14), (150, 10, 0, 170, 20, 9)])
    src = abi.reference_source(sx=100.3, sy=12.2, sz=10.1, ex=100.3, ey=12.2, ez=10.1, amp=1e-3, t0=12.0,
                               sigma_t=3.0)
    probes = np.array([[110.5, 12.5, 10.5], [90.5, 8.5, 6.5], [128.5, 12.5, 10.5], [64.5, 20.5, 3.5],
                       [150.5, 5.5, 12.5], [60.5, 12.5, 10.5]])
    return dict(cfg=cfg, sources=[src], probes=probes, triangles=tris, steps=steps)


def fp16_case(name):
    if name == "wide_box":
        return wide_box()
    amp = {"scatter_small": 1e-3, "lloyd_small": 5e-4, "city_small": 1e-3}[name]
    sc = scenarios.scenario(name, storage=abi.LBM_STORE_F16, f16_scale=1.0 / amp)
    sc["steps"] = min(sc["steps"], 120)
    return sc


def run(sc):
    g = nlos_lbm.Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(sc["steps"])
    out = g.get_probes(), g.get_rho(), g.get_f()
    g.close()
    return out


@pytest.mark.parametrize("name", ["scatter_small", "lloyd_small", "city_small", "wide_box"])
def test_fp16_step_matches_oracle(name, gpu):
    sc = fp16_case(name)
    probes, _, _ = run(sc)
    assert np.max(np.abs(probes)) > 0
    o = oracle.OracleSolver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    o.step(sc["steps"])
    assert rel_l2(probes, o.get_probes()) <= FP16_PROBE_TOL, rel_l2(probes, o.get_probes())


def test_fp16_step_is_deterministic(gpu):
    sc = fp16_case("city_small")
    a, b = run(sc), run(sc)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def odd_box(n3, storage, steps=30):
    """Open box (NSCBC on every face) of an odd shape: rows shorter than, equal
    to, or just longer than a 64-cell block, single-row planes."""
    nx, ny, nz = n3
    cfg = scenarios.lattice_config(nx, ny, nz, 0.55, face_bc=(abi.LBM_BC_NSCBC,) * 6, sponge_faces=0,
                                   storage=storage, f16_scale=1000.0)
    c = (nx / 2 + 0.1, ny / 2 + 0.2, nz / 2 + 0.3)
    src = abi.reference_source(sx=c[0], sy=c[1], sz=c[2], ex=c[0], ey=c[1], ez=c[2], amp=1e-3, t0=6.0,
                               sigma_t=2.0)
    probes = np.array([[0.5, 0.5, 0.5], [nx - 0.5, ny - 0.5, nz - 0.5], [min(c[0] + 1.0, nx - 0.5), c[1], c[2]],
                       [min(nx - 0.5, 63.5), 0.5, nz - 0.5]])
    return dict(cfg=cfg, sources=[src], probes=probes, triangles=None, steps=steps)


ODD_SHAPES = [(1, 5, 4), (3, 2, 3), (63, 2, 2), (65, 3, 2), (130, 1, 3)]


@pytest.mark.parametrize("n3", ODD_SHAPES)
def test_odd_shapes_match_oracle(n3, gpu):
    sc32 = odd_box(n3, abi.LBM_STORE_F32)
    o = oracle.OracleSolver(sc32["cfg"], sc32["sources"], sc32["probes"])
    o.step(sc32["steps"])
    ref = o.get_probes()
    assert np.max(np.abs(ref)) > 0
    g = nlos_lbm.Solver(sc32["cfg"], sc32["sources"], sc32["probes"])
    g.step(sc32["steps"])
    assert rel_l2(g.get_probes(), ref) <= 1e-5, rel_l2(g.get_probes(), ref)
    sc16 = odd_box(n3, abi.LBM_STORE_F16)
    probes, _, _ = run(sc16)
    assert rel_l2(probes, ref) <= FP16_PROBE_TOL, (n3, rel_l2(probes, ref))
