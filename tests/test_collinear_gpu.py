"""Collinear spin functional on the device (sdft_b200_collinear_functionals).

Against the reference's evaluate_collinear_density_functionals
(tests/golden/collinear_*.npz, up and down Gaussian densities with different
supports, with and without a frozen core split between the channels): the
bars of test_oracle_pins.check_collinear (energies, electrons and
<n_s, v_xc,s> 1e-12 relative, stresses 1e-11, minimum 1e-10, counts of
negative samples exact, potentials 1e-11, or 1e-6 where floored samples make
the reference's own response ill-conditioned). At the Si64 scale (142^3 = 2 x
71 per axis) the nonmagnetic limit n_up = n_down = n/2 reproduces the
spin-unpolarised functional: total XC energy within 1e-10 relative, each
channel's v_xc and potential within 1e-6 of the unpolarised ones, Hartree
split equally.
"""
import numpy as np
import pytest

from conftest import relative_error
from sdft_b200 import density, synthetic
from test_oracle_pins import COLLINEAR_POTENTIAL_TOL, check_collinear, collinear_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["si8", "triclinic"])
@pytest.mark.parametrize("label", ["plain", "core"])
def test_collinear_matches_reference(context, golden, name, label):
    case, core = collinear_inputs(name, label)
    result = density.collinear_functionals(context, case["lattice"], case["up_keys"], case["up"], case["down_keys"],
                                           case["down"], core.get("core_hkl"), core.get("core"))
    check_collinear(result, golden(f"collinear_{name}"), label, COLLINEAR_POTENTIAL_TOL[name])


def test_nonmagnetic_limit_is_the_unpolarised_functional(context):
    c = synthetic.functional_case("si64")
    half = 0.5 * c["values"]
    spin = density.collinear_functionals(context, c["lattice"], c["keys"], half, c["keys"], half)
    plain = density.density_functionals(context, c["lattice"], c["keys"], c["values"])
    assert spin["up"]["grid"] == plain["grid"] == (142, 142, 142)
    assert np.array_equal(spin["hkl"], plain["hkl"])
    total_xc = spin["up"]["xc_energy"] + spin["down"]["xc_energy"]
    assert abs(total_xc - plain["xc_energy"]) <= 1e-10 * abs(plain["xc_energy"])
    assert abs(2 * spin["up"]["hartree_energy"] - plain["hartree_energy"]) <= 1e-12 * plain["hartree_energy"]
    for channel in ("up", "down"):
        assert relative_error(spin[channel]["xc_potential"], plain["xc_potential"]) < 1e-6
        assert relative_error(spin[channel]["potential"], plain["potential"]) < 1e-6
    assert relative_error(spin["up"]["xc_potential"], spin["down"]["xc_potential"]) < 1e-12


def test_collinear_host_checks(context):
    c = synthetic.collinear_case("triclinic")
    with pytest.raises(ValueError, match="invalid collinear density/lattice"):
        density.collinear_functionals(context, np.zeros((3, 3)), c["up_keys"], c["up"], c["down_keys"], c["down"])
    with pytest.raises(ValueError, match="invalid collinear XC padding"):
        density.collinear_functionals(context, c["lattice"], c["up_keys"], c["up"], c["down_keys"], c["down"],
                                      padding=9)
    bad = c["up"].copy()
    bad[0] = np.nan
    with pytest.raises(ValueError, match="nonfinite spin density"):
        density.collinear_functionals(context, c["lattice"], c["up_keys"], bad, c["down_keys"], c["down"])
