"""Hartree + PBE functional on the device (sdft_b200_density_functionals).

Bars against the reference's evaluate_density_functionals
(tests/golden/functional_*.npz, seeded Gaussian densities on prime-length
grids, without and with a frozen core): 1e-12 relative on the Hartree and XC
energies, electrons and <n, v_xc>, 1e-11 relative on the stresses and the
potentials (PBE point arithmetic from CUDA's libm differs from the host's in
the last bits), the minimum density 1e-10, the clipped count exact. At the
Si64 scale (f = 4 support, 191 711 keys, grid 142^3 = 2 x 71 per axis) the
numpy oracle is the checker with the same bars, plus properties that hold at
any size: the Hartree part equals 4 pi n / q^2, the sampled electrons equal
Omega n(0), v_xc is Hermitian, and a translation by one grid step moves v_xc
by its phase and leaves the XC energy unchanged.
"""
import os

import numpy as np
import pytest

from conftest import relative_error
from oracle import sdft_oracle
from sdft_b200 import density, synthetic
from test_oracle_pins import check_functional, functional_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["si8", "triclinic"])
@pytest.mark.parametrize("label", ["plain", "core"])
def test_functional_matches_reference(context, golden, name, label):
    case, core = functional_inputs(name, label)
    result = density.density_functionals(context, case["lattice"], case["keys"], case["values"],
                                         core.get("core_keys"), core.get("core_values"))
    check_functional(result, golden(f"functional_{name}"), label, 1e-12, 1e-11)


@pytest.fixture(scope="module")
def si64_case():
    return synthetic.functional_case("si64")


@pytest.fixture(scope="module")
def si64_device(context, si64_case):
    c = si64_case
    return density.density_functionals(context, c["lattice"], c["keys"], c["values"], c["core_keys"],
                                       c["core_values"])


def test_si64_functional_matches_oracle(si64_case, si64_device):
    c = si64_case
    o = sdft_oracle.density_functionals(c["lattice"], c["keys"], c["values"], c["core_keys"], c["core_values"])
    d = si64_device
    assert d["grid"] == (142, 142, 142) and o["grid"] == d["grid"]
    assert np.array_equal(d["hkl"], o["hkl"])
    for name in ("hartree_energy", "xc_energy", "vxc_density", "sampled_electrons"):
        assert abs(d[name] - o[name]) <= 1e-12 * abs(o[name]), name
    for name in ("hartree_stress", "xc_stress"):
        assert np.max(np.abs(d[name] - o[name])) <= 1e-11 * np.max(np.abs(o[name])), name
    assert abs(d["minimum_density"] - o["minimum_density"]) <= 1e-10 * abs(o["minimum_density"])
    assert d["clipped_density_points"] == o["clipped_density_points"]
    for name in ("potential", "xc_potential"):
        assert relative_error(d[name], o[name]) < 1e-11, name


def test_si64_functional_properties(si64_case, si64_device):
    c, d = si64_case, si64_device
    lattice = np.asarray(c["lattice"])
    volume = abs(np.linalg.det(lattice))
    b = 2 * np.pi * np.linalg.inv(lattice).T
    where = {tuple(k): i for i, k in enumerate(d["hkl"].tolist())}
    rows = np.array([where[tuple(k)] for k in c["keys"].tolist()])
    q = c["keys"].astype(np.float64) @ b
    q2 = (q * q).sum(axis=1)
    hartree = np.where(q2 > 1e-12, 4 * np.pi * c["values"] / np.where(q2 > 1e-12, q2, 1.0), 0.0)
    assert relative_error(d["potential"][rows] - d["xc_potential"][rows], hartree) < 1e-14
    density_zero = c["values"][np.flatnonzero((c["keys"] == 0).all(axis=1))[0]].real
    assert abs(d["sampled_electrons"] - volume * density_zero) <= 1e-12 * volume * density_zero
    opposite = np.array([where[(-h, -k, -l)] for h, k, l in d["hkl"].tolist()])
    assert relative_error(d["xc_potential"][opposite], np.conj(d["xc_potential"])) < 1e-12


def test_translation_by_a_grid_step(context, si64_case, si64_device):
    """Shifting every site by one XC grid step along a1 multiplies n(G) and
    v_xc(G) by exp(-2 pi i h / n0) and leaves the XC energy unchanged (the
    grid samples the shifted density at the same values)."""
    c, d = si64_case, si64_device
    n0 = d["grid"][0]
    phase = np.exp(-2j * np.pi * c["keys"][:, 0] / n0)
    core_phase = np.exp(-2j * np.pi * c["core_keys"][:, 0] / n0)
    shifted = density.density_functionals(context, c["lattice"], c["keys"], c["values"] * phase, c["core_keys"],
                                          c["core_values"] * core_phase)
    assert abs(shifted["xc_energy"] - d["xc_energy"]) <= 1e-12 * abs(d["xc_energy"])
    assert abs(shifted["hartree_energy"] - d["hartree_energy"]) <= 1e-12 * abs(d["hartree_energy"])
    support_phase = np.exp(-2j * np.pi * d["hkl"][:, 0] / n0)
    assert relative_error(shifted["xc_potential"], d["xc_potential"] * support_phase) < 1e-11


def test_fast_grid_and_padding_match_oracle(context):
    case = synthetic.functional_case("si8")
    for padding, fast in ((1, False), (3, False), (2, True)):
        os.environ["SDFT_FAST_DENSITY_GRID"] = "1" if fast else "0"
        try:
            d = density.density_functionals(context, case["lattice"], case["keys"], case["values"],
                                            quadrature_padding=padding)
        finally:
            del os.environ["SDFT_FAST_DENSITY_GRID"]
        o = sdft_oracle.density_functionals(case["lattice"], case["keys"], case["values"], padding=padding, fast=fast)
        assert d["grid"] == o["grid"], (padding, fast)
        assert abs(d["xc_energy"] - o["xc_energy"]) <= 1e-12 * abs(o["xc_energy"])
        assert relative_error(d["potential"], o["potential"]) < 1e-11
