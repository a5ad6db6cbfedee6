"""Pins the oracle: numpy restatement vs the reference's own outputs (CPU only)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import probe_block, relative_error
from oracle import ref_oracle, sdft_oracle
from sdft_b200 import synthetic


@pytest.mark.parametrize("binary,marker", [
    ("plane_wave_operator_smoke", "plane_wave_operator PASS"),
    ("fft_backend_smoke", '"passed":true'),
    ("davidson_optimization_smoke", "PASS"),
])
def test_reference_smoke_tests_pass_with_shims(binary, marker, tmp_path):
    """The reference's own oracle tests (dense assembly, convolution, dense eigensolver) pass on this build."""
    path = ref_oracle.HERE / "_ref" / binary
    if not path.exists():
        pytest.skip("reference smoke binaries not built")
    env = dict(os.environ, OMP_NUM_THREADS="4", OPENBLAS_NUM_THREADS="1")
    run = subprocess.run([str(path)], cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    assert marker in run.stdout


@pytest.mark.parametrize("name,factory", [("tiny", synthetic.tiny), ("si8", synthetic.si8)])
def test_metric_signature_decisions_match_reference(reference, name, factory):
    """The numpy restatement of overlap()'s signature block reaches the
    reference's decision on a definite, a singular and an indefinite S~
    (src/plane_wave_operator.cpp:702-717)."""
    x = factory()
    minimum, indefinite, singular = sdft_oracle.metric_signature(sdft_oracle.Operator(x))
    assert abs(minimum - 0.3) < 1e-12 and not indefinite and not singular  # the generator's lambda_min(S~) = 0.3
    assert not ref_oracle.ReferenceOperator(reference, x).overlap_signature()["indefinite"]
    pencil = synthetic.scaled_overlap(x, synthetic.singular_overlap_factor(minimum, x.regularization))
    m, indefinite, singular = sdft_oracle.metric_signature(sdft_oracle.Operator(pencil))
    assert singular and not indefinite and abs(m) < 1e-13
    with pytest.raises(RuntimeError, match="original PAW overlap is numerically singular"):
        ref_oracle.ReferenceOperator(reference, pencil).overlap_signature()
    pencil = synthetic.scaled_overlap(x, 1.5)
    m, indefinite, singular = sdft_oracle.metric_signature(sdft_oracle.Operator(pencil))
    assert indefinite and not singular and m < -0.01
    assert ref_oracle.ReferenceOperator(reference, pencil).overlap_signature()["indefinite"]


@pytest.mark.parametrize("name,factory", [("tiny", synthetic.tiny), ("si8", synthetic.si8)])
def test_enumeration_bit_exact_against_golden(golden, name, factory):
    g = golden(name)
    x = factory()
    assert np.array_equal(x.hkl, g["hkl"])
    assert np.array_equal(x.kinetic_ev, g["kinetic_ev"])


@pytest.mark.parametrize("name,factory", [("tiny", synthetic.tiny), ("si8", synthetic.si8)])
def test_numpy_operator_matches_reference(golden, name, factory):
    g = golden(name)
    x = factory()
    op = sdft_oracle.Operator(x)
    assert tuple(op.shape) == tuple(g["shape"])
    assert np.array_equal(op.indices, g["indices"])
    assert np.array_equal(op.kinetic, g["kinetic"])
    assert relative_error(op.local_real, g["local_real"]) < 1e-13
    assert relative_error(op.h_diagonal, g["h_diagonal"]) < 1e-13
    assert relative_error(op.s_diagonal, g["s_diagonal"]) < 1e-13
    probe = probe_block(x.npw, 4, int(g["probe_seed"]))
    assert relative_error(op.apply_h(probe), g["hx"]) < 1e-12
    assert relative_error(op.apply_s(probe), g["sx"]) < 1e-12


def test_dense_eigenvalues_match_reference_davidson(golden, tiny_inputs):
    g = golden("tiny")
    op = sdft_oracle.Operator(tiny_inputs)
    h, s = op.dense()
    values = sdft_oracle.generalized_eigenvalues(h, s, tiny_inputs.roots)
    assert bool(g["converged"])
    assert np.max(np.abs(values - g["eigenvalues"])) < 1e-10
    assert np.max(g["residuals"]) <= 1e-12


def test_golden_solutions_are_certified(golden):
    for name in ("tiny", "si8"):
        g = golden(name)
        assert bool(g["converged"]) and np.max(g["residuals"]) <= 1e-12


def test_kinetic_preconditioner_matches_reference(reference):
    for t in (0.0, 1e-3, 0.05, 0.7, 3.0, 15.0, 400.0):
        for wk in (0.0, 0.01, 0.5, 2.0):
            assert sdft_oracle.kinetic_preconditioner(t, wk) == reference.kinetic_preconditioner(t, wk)


def test_live_reference_reproduces_golden(reference, golden, tiny_inputs):
    g = golden("tiny")
    op = ref_oracle.ReferenceOperator(reference, tiny_inputs)
    probe = probe_block(tiny_inputs.npw, 4, int(g["probe_seed"]))
    assert relative_error(op.apply(probe, overlap=False), g["hx"]) < 1e-14
    hkl, _, kin = reference.enumerate_g_vectors(tiny_inputs.reciprocal, tiny_inputs.ecut_ha * synthetic.HARTREE_TO_EV)
    assert np.array_equal(hkl, tiny_inputs.hkl) and np.array_equal(kin, tiny_inputs.kinetic_ev)


def test_kpoint_enumeration_bit_exact(reference):
    x = synthetic.tiny()
    for k in ((1 / 3, 0.0, -1 / 3), (0.25, 0.5, 0.0)):
        hkl, cart, kin = synthetic.enumerate_g_vectors(x.reciprocal, 4.0 * synthetic.HARTREE_TO_EV, k)
        rh, rc, rk = reference.enumerate_g_vectors(x.reciprocal, 4.0 * synthetic.HARTREE_TO_EV, k)
        assert np.array_equal(hkl, rh) and np.array_equal(kin, rk) and np.array_equal(cart, rc)


def test_pbe_restatement_matches_golden(golden):
    g = golden("pbe")
    points = sdft_oracle.pbe_unpolarized(g["density"], g["gradient"])
    scaled = np.abs(points - g["points"]) / np.maximum(1.0, np.abs(g["points"]))
    assert scaled.max() < 1e-14


def test_pbe_restatement_matches_live_reference(reference):
    rng = np.random.Generator(np.random.PCG64(5))
    n = 10.0 ** rng.uniform(-10, 1.5, 4096)
    g = n * rng.uniform(0, 40, 4096)
    ref = reference.pbe(n, g)
    scaled = np.abs(sdft_oracle.pbe_unpolarized(n, g) - ref) / np.maximum(1.0, np.abs(ref))
    assert scaled.max() < 1e-14


@pytest.mark.parametrize("name,factory", [("tiny", synthetic.tiny), ("si8", synthetic.si8)])
def test_band_density_restatement_matches_golden(golden, name, factory):
    g = golden(f"density_{name}")
    x = factory()
    coefficients = synthetic.band_coefficients(x, int(g["bands"]))
    for fast in (False, True):
        out = sdft_oracle.plane_wave_density(x.hkl, coefficients, g["occupations"], x.volume, g["support"], fast)
        assert relative_error(out, g["density"]) < 1e-13


def test_band_density_grid_rule_matches_reference_cases():
    x = synthetic.si8()
    # Span 16 of the Si8 basis dominates a small support: 2*16+1 = 33, rounded to 35.
    assert sdft_oracle.density_grid_shape(x.hkl, synthetic.density_support(x, 2.0)) == (33, 33, 33)
    assert sdft_oracle.density_grid_shape(x.hkl, synthetic.density_support(x, 2.0), fast=True) == (35, 35, 35)
    # min/max are seeded at 0: a basis on one side of the origin still counts from 0.
    hkl = np.array([[2, 3, 4], [5, 3, 4]])
    assert sdft_oracle.density_grid_shape(hkl, np.array([[0, 0, 0]])) == (11, 7, 9)


def test_onsite_and_compensation_restatements_match_golden(golden):
    g = golden("compensation_si8")
    x = synthetic.si8()
    aug = synthetic.augmentation()
    rows = int(np.sum(2 * aug["channel_l"] + 1))
    amplitudes = synthetic.projected_amplitudes(x.positions.shape[0], rows, int(g["bands"]))
    onsite = np.stack([sdft_oracle.onsite_density(amplitudes[a * rows:(a + 1) * rows], g["occupations"])
                       for a in range(x.positions.shape[0])])
    assert relative_error(onsite, g["onsite"]) < 1e-14
    # The synthetic (L,M) transform (Gaunt coefficients by quadrature) is the reference's.
    assert np.max(np.abs(synthetic.lm_transform(aug) - g["transform"])) < 1e-14
    keys = synthetic.density_support(x, float(g["factor"]))
    charge = sdft_oracle.compensation_density(x.lattice, x.positions, keys, aug, g["transform"], g["onsite"])
    assert relative_error(charge, g["charge"]) < 1e-13


def test_compensation_restatement_matches_live_reference_off_gamma_lattice(reference):
    """A non-cubic cell and a complex (non-real) occupation, against the reference itself."""
    rng = np.random.Generator(np.random.PCG64(3))
    lattice = np.array([[6.0, 0.4, 0.0], [0.3, 7.0, 0.2], [0.0, -0.5, 6.5]])
    fractional = rng.uniform(0, 1, (3, 3))
    keys = np.array([(h, k, l) for h in range(-4, 5) for k in range(-4, 5) for l in range(-4, 5)], dtype=np.int32)
    aug = synthetic.augmentation(seed=5)
    m = rng.standard_normal((3, 8, 8)) + 1j * rng.standard_normal((3, 8, 8))
    onsite = m + np.conj(np.transpose(m, (0, 2, 1)))
    expected = reference.compensation_density(lattice, fractional, keys, aug, onsite)
    charge = sdft_oracle.compensation_density(lattice, fractional, keys, aug, synthetic.lm_transform(aug), onsite)
    assert relative_error(charge, expected) < 1e-13


def _potential_on_support(keys, potential_keys, potential):
    """V on the support keys in their order, 0 where the potential has no mode."""
    where = {tuple(k): v for k, v in zip(np.asarray(potential_keys).tolist(), potential)}
    return np.array([where.get(tuple(k), 0.0) for k in np.asarray(keys).tolist()], dtype=np.complex128)


def test_compensation_projection_restatement_matches_golden(golden):
    """The adjoint (project_potential_batch) against the reference's fixture:
    a potential missing 2 % of the support's modes and carrying modes outside it."""
    g = golden("compensation_project_si8")
    x = synthetic.si8()
    aug = synthetic.augmentation()
    keys = synthetic.density_support(x, float(g["factor"]))
    v = _potential_on_support(keys, g["potential_keys"], g["potential"])
    out = sdft_oracle.compensation_project(x.lattice, x.positions, keys, aug, synthetic.lm_transform(aug), v)
    assert relative_error(out, g["projection"]) < 1e-12


FUNCTIONAL_SCALARS = ("hartree_energy", "xc_energy", "vxc_density", "sampled_electrons")


def functional_inputs(name, label):
    case = synthetic.functional_case(name)
    core = {"core_keys": case["core_keys"], "core_values": case["core_values"]} if label == "core" else {}
    return case, core


def check_functional(result, golden, label, scalar_tol, potential_tol):
    """Shared bars for the functional: keys in the same order, scalars and
    stresses relative, the minimum density relative, the clipped count exact,
    potentials relative in norm."""
    assert np.array_equal(np.asarray(result["hkl"]), golden[f"{label}_hkl"])
    assert int(result["grid_points"]) == int(golden[f"{label}_grid_points"])
    for name in FUNCTIONAL_SCALARS:
        expected = float(golden[f"{label}_{name}"])
        assert abs(result[name] - expected) <= scalar_tol * abs(expected), name
    for name in ("hartree_stress", "xc_stress"):
        expected = golden[f"{label}_{name}"]
        assert np.max(np.abs(np.asarray(result[name]) - expected)) <= 10 * scalar_tol * np.max(np.abs(expected)), name
    expected_min = float(golden[f"{label}_minimum_density"])
    assert abs(result["minimum_density"] - expected_min) <= 1e-10 * abs(expected_min)
    assert int(result["clipped_density_points"]) == int(golden[f"{label}_clipped_density_points"])
    for name in ("potential", "xc_potential"):
        assert relative_error(result[name], golden[f"{label}_{name}"]) < potential_tol, name


@pytest.mark.parametrize("name", ["si8", "triclinic"])
@pytest.mark.parametrize("label", ["plain", "core"])
def test_functional_restatement_matches_golden(golden, name, label):
    """The numpy restatement of evaluate_density_functionals against the
    reference's outputs (tests/golden/functional_*.npz): 1e-12 relative on
    energies, electrons and <n, v_xc>, 1e-12 on the potentials."""
    case, core = functional_inputs(name, label)
    result = sdft_oracle.density_functionals(case["lattice"], case["keys"], case["values"], **core)
    check_functional(result, golden(f"functional_{name}"), label, 1e-12, 1e-12)


def test_functional_restatement_matches_live_reference_padding(reference):
    """Quadrature padding 1 and 3 (the reference's override), against the live reference."""
    case = synthetic.functional_case("triclinic")
    for padding in (1, 3):
        r = reference.density_functionals(case["lattice"], case["keys"], case["values"], padding=padding)
        o = sdft_oracle.density_functionals(case["lattice"], case["keys"], case["values"], padding=padding)
        assert r["grid_points"] == o["grid_points"]
        assert abs(r["xc_energy"] - o["xc_energy"]) <= 1e-12 * abs(r["xc_energy"])
        assert relative_error(o["potential"], r["potential"]) < 1e-12


# Potential bars of the collinear form: Si8's channels have samples at the
# 5e-11 density floor where the gradient is rounding noise (|grad n| ~ 1e-17)
# times a large dE/dsigma, so a 1e-16 relative change of the real-space fields
# moves the gradient response by ~1e-5 there and the potential by ~1e-7 in
# norm, in the reference's own formula; the triclinic case has no such points.
COLLINEAR_POTENTIAL_TOL = {"si8": 1e-6, "triclinic": 1e-11}


def collinear_inputs(name, label):
    case = synthetic.collinear_case(name)
    core = {"core_hkl": case["core_keys"], "core": case["core_values"]} if label == "core" else {}
    return case, core


def check_collinear(result, golden, label, potential_tol):
    assert np.array_equal(np.asarray(result["hkl"]), golden[f"{label}_hkl"])
    for channel in ("up", "down"):
        r = result[channel]
        g = {k[len(label) + len(channel) + 2:]: v for k, v in golden.items() if k.startswith(f"{label}_{channel}_")}
        assert int(r["grid_points"]) == int(g["grid_points"])
        for name in ("hartree_energy", "xc_energy", "vxc_density", "sampled_electrons"):
            assert abs(r[name] - float(g[name])) <= 1e-12 * max(abs(float(g[name])), 1e-300), (channel, name)
        for name in ("hartree_stress", "xc_stress"):
            assert np.max(np.abs(np.asarray(r[name]) - g[name])) <= 1e-11 * np.max(np.abs(g[name])), (channel, name)
        assert abs(r["minimum_density"] - float(g["minimum_density"])) <= 1e-10 * abs(float(g["minimum_density"]))
        assert int(r["clipped_density_points"]) == int(g["clipped_density_points"])
        for name in ("potential", "xc_potential"):
            assert relative_error(r[name], g[name]) < potential_tol, (channel, name)


@pytest.mark.parametrize("name", ["si8", "triclinic"])
@pytest.mark.parametrize("label", ["plain", "core"])
def test_collinear_restatement_matches_golden(golden, name, label):
    """The numpy restatement of evaluate_collinear_density_functionals against
    the reference's outputs (tests/golden/collinear_*.npz)."""
    case, core = collinear_inputs(name, label)
    result = sdft_oracle.collinear_functionals(case["lattice"], case["up_keys"], case["up"], case["down_keys"],
                                               case["down"], core.get("core_hkl"), core.get("core"))
    check_collinear(result, golden(f"collinear_{name}"), label, COLLINEAR_POTENTIAL_TOL[name])


def test_spin_pbe_restatement_matches_live_reference(reference):
    """The numpy restatement of pbe_collinear (src/spin_pbe_xc.cpp:54-107)
    against the reference per point: densities over 12 decades, polarisation
    from unpolarised to the zeta clamp, random gradients; energies and
    potentials to 1e-12 relative, gradient responses to 1e-11 of each point's
    scale."""
    rng = np.random.Generator(np.random.PCG64(5))
    count = 4000
    total = np.exp(rng.uniform(np.log(1e-8), np.log(1e4), count))
    zeta = rng.uniform(-1.0, 1.0, count)
    zeta[:40] = 0.0
    zeta[40:80] = np.sign(zeta[40:80]) * (1 - 1e-14)
    up = np.maximum(0.5 * total * (1 + zeta), 5e-11)
    down = np.maximum(0.5 * total * (1 - zeta), 5e-11)
    gu = rng.standard_normal((count, 3)) * up[:, None] ** (4.0 / 3.0)
    gd = rng.standard_normal((count, 3)) * down[:, None] ** (4.0 / 3.0)
    expected = reference.pbe_collinear(up, down, gu, gd)
    energy, potentials, response = sdft_oracle.pbe_collinear(up, down, gu, gd)
    assert np.max(np.abs(energy - expected[:, 0]) / np.maximum(np.abs(expected[:, 0]), 1e-300)) < 1e-12
    for s in range(2):
        v = expected[:, 1 + s]
        assert np.max(np.abs(potentials[s] - v) / np.maximum(np.abs(v), 1e-300)) < 1e-12
        r = expected[:, 3 + 3 * s:6 + 3 * s]
        scale = np.maximum(np.abs(r).max(axis=1, keepdims=True), 1e-300)
        assert np.max(np.abs(response[s] - r) / scale) < 1e-11
