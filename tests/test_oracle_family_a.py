"""The oracle's scheme-A (family 01-04) restatement against the unmodified
01_acoustic_scattering.cpp, 02_lloyds_mirror.cpp, 03_doppler_effect.cpp and
04_hpc_scalability.cpp (built by oracle/Makefile's
`ref` target through oracle/ref_harness_a.cpp where the reference sources
are present) and against the fixtures they produced (tests/golden, always).

Measured agreement: 01 and 03 bit-identical; 04 within 2.4e-13 of the
field's largest deviation (its source term is summed in another order); 02 within 1e-14 of the field's
largest deviation, from the source weight written as exp(-r^2/(2 sigma^2))
instead of 02's exp(-ln2 r^2/b) with the same width.  Bound: 1e-12.
"""
import os

import numpy as np
import pytest

import oracle
import scenarios
from oracle import OracleSolver

TOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _oracle_rho(sc):
    o = OracleSolver(sc["cfg"], sc["sources"], sc["probes"], mask=sc["mask"], blend_xy=sc.get("blend_xy"),
                     field_xy=sc.get("field_xy"))
    if sc.get("rho0") is not None:
        o.set_density(sc["rho0"])
    o.step(sc["steps"])
    nx, ny, nz = o.dims_halo
    rho = o.get_rho().reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1] - 1.0
    mask = o.get_mask().reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1]
    rho[mask == 1] = 0.0
    return o, rho


@pytest.mark.parametrize("name", ["lloyd_a", "doppler_a", "scattering_a", "hpc_a"])
def test_oracle_matches_family_a_fixture(name):
    gold = np.load(os.path.join(GOLDEN, name + ".npz"))
    sc = scenarios.family_a(name, steps=int(gold["steps"]))
    o, rho = _oracle_rho(sc)
    assert tuple(gold["dims_halo"]) == o.dims_halo
    assert o.dt == float(gold["dt"])
    assert np.array_equal(np.packbits(o.get_mask()), gold["mask_bits"])
    ref = gold["rho_minus_1"]
    assert np.max(np.abs(ref)) > 1e-6
    assert np.max(np.abs(rho - ref)) <= TOL * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["lloyd_a", "doppler_a", "scattering_a", "hpc_a"])
def test_oracle_matches_family_a_reference(name):
    sc = scenarios.family_a(name, steps=25)
    if not oracle.refa_available(sc["ref"]):
        pytest.skip("reference family-A harness not built here")
    ref = oracle.RefASolver(sc["ref"], **sc["ref_params"])
    o, rho = _oracle_rho(sc)
    mask = ref.get_mask()
    fluid = mask == 0
    assert np.array_equal(mask, o.get_mask())
    assert np.max(np.abs(ref.get_tau()[fluid] - o.get_tau_a()[fluid])) <= 1e-15
    if sc["cfg"].sponge_blend:
        # interior cells (04 also fills its halo cells, which are never updated)
        nx, ny, nz = ref.dims_halo
        inner = (slice(1, -1),) * 3
        fi = fluid.reshape(nz, ny, nx)[inner]
        sr, so = ref.get_sponge().reshape(nz, ny, nx)[inner], o.get_sponge().reshape(nz, ny, nx)[inner]
        assert np.max(np.abs(sr[fi] - so[fi])) <= 1e-15
    ref.step(sc["steps"])
    nx, ny, nz = ref.dims_halo
    rr = ref.get_rho().reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1] - 1.0
    rr[mask.reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1] == 1] = 0.0
    assert np.max(np.abs(rho - rr)) <= TOL * np.max(np.abs(rr))


def test_scattering_workload_matches_reference_setup():
    """The full-size 01 workload (bench) builds 01's own mask, initial
    density and sponge: checked against 01's init_physics at its own size."""
    if not oracle.refa_available("01"):
        pytest.skip("reference family-A harness not built here")
    from nlos_lbm import workloads

    w = workloads.build("scattering_a")
    ref = oracle.RefASolver("01", x_min=-8.0, x_max=8.0, y_min=-8.0, y_max=8.0, z_min=-0.2, z_max=0.2, dx=0.05,
                            amp=0.01)
    nx, ny, nz = ref.dims_halo
    assert (nx - 2, ny - 2, nz - 2) == workloads.cells(w["cfg"])
    mask = ref.get_mask()
    assert np.array_equal(mask, w["mask"])
    inner = (slice(1, -1),) * 3
    rr = ref.get_rho().reshape(nz, ny, nx)[inner] - 1.0
    rr[mask.reshape(nz, ny, nx)[inner] == 1] = 0.0
    assert np.max(np.abs(rr.ravel() - w["rho0"])) <= 1e-15
    o = OracleSolver(w["cfg"], w["sources"], w["probes"], mask=w["mask"])
    fluid = mask == 0
    assert np.max(np.abs(ref.get_sponge()[fluid] - o.get_sponge()[fluid])) <= 1e-15
