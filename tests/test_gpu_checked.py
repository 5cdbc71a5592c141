"""The bounds-checked library (liblbm_b200_check.so, NLOS_LBM_CHECK=1) on the
GPU: its self-test trips exactly one check, and the forward (FP32, FP16 warp
pipelines), scheme-A (03, and 01 with its blend sponge,
periodic z and initial density) and adjoint kernels run the parity
scenarios without a single out-of-range index, with the same results as the
product library.  The checked library runs in a child process (a process
loads one of the two libraries)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from nlos_lbm import LBMError, Solver, abi

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, os, sys
sys.path[:0] = [sys.argv[1], os.path.join(sys.argv[1], "city-scale-nlos-acoustic-engine-code_b200"),
                os.path.join(sys.argv[1], "tests")]
import numpy as np
import scenarios
from nlos_lbm import Solver, abi
import test_gpu_fp16_step as tv
assert abi.CHECKED
out = {}
sc = scenarios.scenario("lloyd_small")
g = Solver(sc["cfg"], sc["sources"], sc["probes"])
g.check_selftest()
out["selftest"] = g.check_status()
out["after_selftest"] = g.check_status()
runs = {
    "fp32_city": scenarios.scenario("city_small"),
    "fp16_city": scenarios.scenario("city_small", storage=abi.LBM_STORE_F16, f16_scale=1e3),
    "fp16_wide": tv.wide_box(),
    "scheme_a": scenarios.family_a("doppler_a", steps=20),
    "scheme_a_01": scenarios.scattering_a(steps=20),
}
for name, s in runs.items():
    g = Solver(s["cfg"], s["sources"], s["probes"], triangles=s.get("triangles"), mask=s.get("mask"))
    if s.get("rho0") is not None:
        g.set_density(s["rho0"])
    g.step(min(s["steps"], 60))
    out[name] = {"status": g.check_status(), "probes": g.get_probes().tolist()}
a = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=30, nprobe=6)
g = Solver(a["cfg"], [a["trial"]], a["probes"], triangles=a["triangles"])
L, gp, gs, _ = g.adjoint_grad(a["observed"], 10, 0)
out["adjoint"] = {"status": g.check_status(), "loss": L, "grad_pos": list(gp)}
print(json.dumps(out))
'''


def _product_runs():
    import scenarios
    import test_gpu_fp16_step as tv

    runs = {
        "fp32_city": scenarios.scenario("city_small"),
        "fp16_city": scenarios.scenario("city_small", storage=abi.LBM_STORE_F16, f16_scale=1e3),
        "fp16_wide": tv.wide_box(),
        "scheme_a": scenarios.family_a("doppler_a", steps=20),
        "scheme_a_01": scenarios.scattering_a(steps=20),
    }
    out = {}
    for name, s in runs.items():
        g = Solver(s["cfg"], s["sources"], s["probes"], triangles=s.get("triangles"), mask=s.get("mask"))
        if s.get("rho0") is not None:
            g.set_density(s["rho0"])
        g.step(min(s["steps"], 60))
        out[name] = g.get_probes()
    a = scenarios.adjoint_scenario(nx=32, ny=24, nz=16, steps=30, nprobe=6)
    g = Solver(a["cfg"], [a["trial"]], a["probes"], triangles=a["triangles"])
    L, gp, _, _ = g.adjoint_grad(a["observed"], 10, 0)
    out["adjoint"] = (L, np.asarray(gp))
    return out


def test_checked_build_finds_no_out_of_range_index(gpu):
    env = dict(os.environ, NLOS_LBM_CHECK="1")
    r = subprocess.run([sys.executable, "-c", CHILD, REPO], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["selftest"] == [99, 37]          # lbm::kChkSelfTest, the index one past its extent
    assert got["after_selftest"] == [0, 0]      # reading clears it
    for key, v in got.items():
        if key not in ("selftest", "after_selftest"):
            assert v["status"] == [0, 0], (key, v["status"])
    ref = _product_runs()
    for name in ("fp32_city", "fp16_city", "fp16_wide", "scheme_a", "scheme_a_01"):
        assert np.array_equal(np.asarray(got[name]["probes"]), ref[name]), name
    assert got["adjoint"]["loss"] == ref["adjoint"][0]
    assert np.array_equal(np.asarray(got["adjoint"]["grad_pos"]), ref["adjoint"][1])


def test_product_build_has_no_checks(gpu):
    import scenarios

    sc = scenarios.scenario("lloyd_small")
    g = Solver(sc["cfg"], sc["sources"], sc["probes"])
    with pytest.raises(LBMError) as e:
        g.check_status()
    assert e.value.status == abi.LBM_ERR_UNSUPPORTED
