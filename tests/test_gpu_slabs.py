"""z-slab decomposition (lbm_config.slab_k0/slab_nz + lbm_slab_exchange),
here with every slab on one GPU: a split run must reproduce the undivided
run.  Bit-identical where no source stencil reaches across a cut (every cell
update reads the same values in the same order); where one does, the
stencil's fluid-weight sum comes from the host in another summation order,
so the bound is 1e-6 of the largest deviation instead."""
import numpy as np
import pytest

import scenarios
from nlos_lbm import LBMError, SlabGroup, Solver, abi

pytestmark = pytest.mark.gpu


def _whole_and_split(sc, nslabs, cuts=None, steps=None):
    steps = steps or sc["steps"]
    g = Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(steps)
    s = SlabGroup(sc["cfg"], nslabs, sc["sources"], sc["probes"], triangles=sc["triangles"], cuts=cuts)
    s.step(steps)
    return g, s


@pytest.mark.parametrize("name,nslabs,cuts", [("ref06_box", 2, [18]), ("scatter_small", 3, None),
                                              ("city_small", 2, [7])])
def test_split_run_is_bit_identical(name, nslabs, cuts, gpu):
    sc = scenarios.scenario(name)
    g, s = _whole_and_split(sc, nslabs, cuts)
    assert np.array_equal(g.get_probes(), s.get_probes(), equal_nan=True)
    assert np.array_equal(g.get_rho(), s.get_rho())


def test_split_fp16_is_bit_identical(gpu):
    sc = scenarios.scenario("scatter_small", storage=abi.LBM_STORE_F16, f16_scale=1e3)
    g, s = _whole_and_split(sc, 2)
    assert np.array_equal(g.get_probes(), s.get_probes(), equal_nan=True)
    assert np.array_equal(g.get_rho(), s.get_rho())


@pytest.mark.parametrize("name,cuts", [("ref06_box", [12, 13]), ("lloyd_small", [10])])
def test_source_across_a_cut(name, cuts, gpu):
    # ref06_box: the 5x5x5 stencil around z = 12.7 spans layers 10-14; lloyd_small:
    # the trilinear source at z = 10 spans layers 9 and 10
    sc = scenarios.scenario(name)
    g, s = _whole_and_split(sc, len(cuts) + 1, cuts, steps=40)
    pg, ps = g.get_probes(), s.get_probes()
    assert np.max(np.abs(pg)) > 0
    assert np.nanmax(np.abs(pg - ps)) <= 1e-6 * np.nanmax(np.abs(pg))
    rg, rs = g.get_rho(), s.get_rho()
    assert np.max(np.abs(rg - rs)) <= 1e-6 * np.max(np.abs(rg))


def test_exchange_rejects_wrong_pairs(gpu):
    sc = scenarios.scenario("ref06_box")
    s = SlabGroup(sc["cfg"], 3, sc["sources"], sc["probes"], triangles=sc["triangles"])
    lib = s.lib
    with pytest.raises(LBMError) as e:
        s.slabs[0]._check(lib.lbm_slab_exchange(s.slabs[0].h, s.slabs[2].h), "x")
    assert e.value.status == abi.LBM_ERR_INVALID_ARGUMENT
    whole = Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    with pytest.raises(LBMError) as e:
        whole._check(lib.lbm_slab_exchange(whole.h, s.slabs[0].h), "x")
    assert e.value.status == abi.LBM_ERR_STATE
