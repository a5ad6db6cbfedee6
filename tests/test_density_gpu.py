"""Density-side kernels on the device against the oracle and the reference's
own fixtures: PBE per point (src/pbe_xc.cpp:119, the sweep and bars of
tests/native/pbe_backend_smoke.cpp)."""
import numpy as np
import pytest

from oracle import sdft_oracle

pytestmark = pytest.mark.gpu

# tests/native/pbe_backend_smoke.cpp:41: every field within 2e-11 scaled by max(1, |ref|),
# central differences of the energy density within 1e-7 of the AD potentials.
PBE_SCALED = 2e-11
PBE_FD = 1e-7


def scaled_error(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def test_pbe_points_match_reference_fixture(context, golden):
    from sdft_b200 import density
    g = golden("pbe")
    out = density.pbe_points(context, g["density"], g["gradient"])
    assert scaled_error(out, g["points"]) < PBE_SCALED


def test_pbe_full_sweep_matches_oracle(context):
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent / "golden"))
    from make_golden import pbe_sampling
    from sdft_b200 import density
    n, g = pbe_sampling()
    out = density.pbe_points(context, n, g)
    assert scaled_error(out, sdft_oracle.pbe_unpolarized(n, g)) < PBE_SCALED


def test_pbe_finite_difference_consistency(context):
    from sdft_b200 import density
    delta = 1e-5
    pn, pg = [], []
    for n in (0.01, 0.1, 0.5, 2.0):
        for g in (0.01, 0.1, 1.0):
            for a, b in ((n, g), (n + delta, g), (n - delta, g), (n, g + delta), (n, g - delta)):
                pn.append(a)
                pg.append(b)
    p = density.pbe_points(context, np.array(pn), np.array(pg))
    worst = 0.0
    for i in range(0, len(pn), 5):
        dn = (p[i + 1, 0] - p[i + 2, 0]) / (2 * delta)
        dg = (p[i + 3, 0] - p[i + 4, 0]) / (2 * delta)
        worst = max(worst, abs(dn - p[i, 4] - p[i, 5]), abs(dg - p[i, 6] * pg[i]))
    assert worst < PBE_FD


@pytest.mark.parametrize("bad", [(0.0, 1.0), (-1.0, 0.0), (1.0, -1e-3), (np.nan, 0.0), (1.0, np.inf)])
def test_pbe_rejects_invalid_points(context, bad):
    from sdft_b200 import _capi, density
    n = np.array([0.3, bad[0], 0.2])
    g = np.array([0.1, bad[1], 0.0])
    with pytest.raises(_capi.InvalidArgument, match="invalid GPU PBE point"):
        density.pbe_points(context, n, g)
    # The context stays usable after the rejected call.
    ok = density.pbe_points(context, np.array([0.3]), np.array([0.1]))
    assert scaled_error(ok, sdft_oracle.pbe_unpolarized([0.3], [0.1])) < PBE_SCALED


def test_pbe_rejects_empty(context):
    from sdft_b200 import _capi, density
    with pytest.raises(_capi.InvalidArgument, match="invalid GPU PBE dimensions"):
        density.pbe_points(context, np.zeros(0), np.zeros(0))


# --- band density (src/density_functionals.cpp:407-460) ------------------------

DENSITY_REL = 1e-12  # FP64 FFTs on a different (smooth) grid: rounding only


def _occupations(bands):
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent / "golden"))
    from make_golden import density_occupations
    return density_occupations(bands)


@pytest.mark.parametrize("name,factory", [("tiny", "tiny"), ("si8", "si8")])
def test_band_density_matches_reference_fixture(context, golden, name, factory):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    g = golden(f"density_{name}")
    x = getattr(synthetic, factory)()
    coefficients = synthetic.band_coefficients(x, int(g["bands"]))
    out = density.band_density(context, x.hkl, coefficients, g["occupations"], x.volume, g["support"])
    assert relative_error(out, g["density"]) < DENSITY_REL


@pytest.mark.parametrize("factor,bands", [(4.0, 32), (8.0, 8), (16.0, 4)])
def test_band_density_si64_matches_oracle(context, factor, bands):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    x = synthetic.si64()
    support = synthetic.density_support(x, factor)
    coefficients = synthetic.band_coefficients(x, bands)
    occ = _occupations(bands)
    out = density.band_density(context, x.hkl, coefficients, occ, x.volume, support)
    expected = sdft_oracle.plane_wave_density(x.hkl, coefficients, occ, x.volume, support, fast=True)
    assert relative_error(out, expected) < DENSITY_REL


def test_band_density_config_size_properties(context):
    """128 bands at f = 16 (density grid 144^3): the G = 0 coefficient equals
    sum_b f_b/Omega for normalised bands (Parseval), n(-G) = conj n(G), and the
    device-memory path returns the host path's values."""
    import torch
    from sdft_b200 import density, synthetic
    x = synthetic.si64()
    support = synthetic.density_support(x, 16.0)
    coefficients = synthetic.band_coefficients(x, 128)
    occ = np.full(128, 2.0)
    out = density.band_density(context, x.hkl, coefficients, occ, x.volume, support)
    zero = int(np.flatnonzero(np.all(support == 0, axis=1))[0])
    assert abs(out[zero] - occ.sum() / x.volume) < 1e-13 * occ.sum() / x.volume
    position = {tuple(k): i for i, k in enumerate(support.tolist())}
    mirror = np.array([position[(-h, -k, -l)] for h, k, l in support.tolist()])
    assert np.max(np.abs(out[mirror] - np.conj(out))) < 1e-15 * np.max(np.abs(out)) * 1e3
    coefficients_device = torch.from_numpy(coefficients).cuda()
    torch.cuda.synchronize()  # the context runs on its own stream: inputs ready before the call
    device = density.band_density(context, x.hkl, coefficients_device, occ, x.volume, support)
    context.synchronize()     # and the result complete before torch reads it
    assert np.array_equal(device.cpu().numpy(), out)


def test_band_density_chunked_bands_match_single_pass(context, monkeypatch):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    x = synthetic.si8()
    support = synthetic.density_support(x, 4.0)
    coefficients = synthetic.band_coefficients(x, 16)
    occ = _occupations(16)
    whole = density.band_density(context, x.hkl, coefficients, occ, x.volume, support)
    monkeypatch.setenv("SDFT_B200_DENSITY_SLAB_BYTES", str(3 * 1024 * 1024))  # a few bands per chunk
    chunked = density.band_density(context, x.hkl, coefficients, occ, x.volume, support)
    assert relative_error(chunked, whole) < 1e-14


def test_band_density_is_linear_in_occupations(context):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    x = synthetic.tiny()
    support = synthetic.density_support(x, 4.0)
    c = synthetic.band_coefficients(x, 3)
    parts = [density.band_density(context, x.hkl, c, np.eye(3)[b] * 2.0, x.volume, support) for b in range(3)]
    occ = np.array([0.5, 2.0, 1.0])
    both = density.band_density(context, x.hkl, c, occ, x.volume, support)
    assert relative_error(both, sum(o / 2.0 * p for o, p in zip(occ, parts))) < 1e-13


def test_band_density_edge_cases(context):
    from sdft_b200 import _capi, density, synthetic
    x = synthetic.tiny()
    support = synthetic.density_support(x, 4.0)
    c = synthetic.band_coefficients(x, 3)
    # All bands empty: zero density, no transform of any band.
    assert not np.any(density.band_density(context, x.hkl, c, np.zeros(3), x.volume, support))
    # A nonfinite coefficient in an empty band is skipped, as in the reference.
    bad = c.copy()
    bad[1, 5] = np.nan
    ok = density.band_density(context, x.hkl, bad, np.array([2.0, 0.0, 2.0]), x.volume, support)
    assert np.all(np.isfinite(ok))
    with pytest.raises(_capi.InvalidArgument, match="nonfinite wavefunction coefficient"):
        density.band_density(context, x.hkl, bad, np.array([2.0, 1.0, 2.0]), x.volume, support)
    for occ in ([2.0, 2.5, 0.0], [2.0, -0.1, 0.0], [np.nan, 1.0, 1.0]):
        with pytest.raises(_capi.InvalidArgument, match="invalid FFT spin-summed occupation"):
            density.band_density(context, x.hkl, c, np.array(occ), x.volume, support)
    for volume in (0.0, -1.0, np.inf):
        with pytest.raises(_capi.InvalidArgument, match="invalid plane-wave FFT density dimensions"):
            density.band_density(context, x.hkl, c, np.ones(3), volume, support)
    with pytest.raises(_capi.InvalidArgument):
        density.band_density(context, x.hkl, c, np.ones(3), x.volume, np.zeros((0, 3), dtype=np.int32))
    dup = x.hkl.copy()
    dup[1] = dup[0]
    with pytest.raises(_capi.InvalidArgument, match="duplicate plane-wave key"):
        density.band_density(context, dup, c, np.ones(3), x.volume, support)
    # The context stays usable after every rejected call.
    again = density.band_density(context, x.hkl, c, np.ones(3), x.volume, support)
    assert np.all(np.isfinite(again))


# --- one-centre occupations and compensation charge ----------------------------

def _compensation_inputs(x, bands, factor):
    from sdft_b200 import synthetic
    aug = synthetic.augmentation()
    rows = int(np.sum(2 * aug["channel_l"] + 1))
    amplitudes = synthetic.projected_amplitudes(x.positions.shape[0], rows, bands)
    return aug, rows, amplitudes, synthetic.density_support(x, factor)


def test_onsite_density_matches_reference_fixture(context, golden):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    g = golden("compensation_si8")
    _, rows, amplitudes, _ = _compensation_inputs(synthetic.si8(), int(g["bands"]), float(g["factor"]))
    onsite = density.onsite_density(context, amplitudes, rows, g["occupations"])
    assert relative_error(onsite, g["onsite"]) < 1e-13


def test_compensation_matches_reference_fixture(context, golden):
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    g = golden("compensation_si8")
    x = synthetic.si8()
    aug, _, _, keys = _compensation_inputs(x, int(g["bands"]), float(g["factor"]))
    charge = density.CompensationCharge(context, x.lattice, x.positions, keys, aug, g["transform"])
    out = charge.density(g["onsite"])
    charge.close()
    assert relative_error(out, g["charge"]) < 1e-12


def test_compensation_si64_f16_matches_oracle_and_device_path(context):
    """Config-size support (Si64, f = 16: ~1.07 M keys, 64 atoms) from 128 occupied bands."""
    import torch
    from conftest import relative_error
    from sdft_b200 import density, synthetic
    x = synthetic.si64()
    aug, rows, amplitudes, keys = _compensation_inputs(x, 128, 16.0)
    occ = np.full(128, 2.0)
    onsite = density.onsite_density(context, amplitudes, rows, occ)
    transform = synthetic.lm_transform(aug)
    charge = density.CompensationCharge(context, x.lattice, x.positions, keys, aug, transform)
    out = charge.density(onsite)
    sub = slice(0, None, 97)  # oracle on a strided subset of the keys
    expected = sdft_oracle.compensation_density(x.lattice, x.positions, keys[sub], aug, transform, onsite)
    assert relative_error(out[sub], expected) < 1e-12
    onsite_device = torch.from_numpy(onsite).cuda()
    torch.cuda.synchronize()
    device = charge.density(onsite_device)
    context.synchronize()
    assert np.array_equal(device.cpu().numpy(), out)
    # n(-G) = conj n(G) for a Hermitian occupation.
    position = {tuple(k): i for i, k in enumerate(keys.tolist())}
    mirror = np.array([position[(-h, -k, -l)] for h, k, l in keys[sub].tolist()])
    assert np.max(np.abs(out[mirror] - np.conj(out[sub]))) < 1e-12 * np.max(np.abs(out))
    charge.close()


def test_onsite_and_compensation_reject_invalid_inputs(context):
    from sdft_b200 import _capi, density, synthetic
    x = synthetic.si8()
    aug, rows, amplitudes, keys = _compensation_inputs(x, 4, 1.0)
    with pytest.raises(_capi.InvalidArgument, match="invalid projected onsite occupation"):
        density.onsite_density(context, amplitudes, rows, [2.0, 2.1, 1.0, 0.0])
    bad = amplitudes.copy()
    bad[3, 1] = np.inf
    with pytest.raises(_capi.InvalidArgument, match="nonfinite onsite projection"):
        density.onsite_density(context, bad, rows, np.ones(4))
    transform = synthetic.lm_transform(aug)
    charge = density.CompensationCharge(context, x.lattice, x.positions, keys, aug, transform)
    onsite = density.onsite_density(context, amplitudes, rows, np.ones(4))
    skew = onsite.copy()
    skew[0, 1, 2] += 1e-6
    with pytest.raises(_capi.InvalidArgument, match="finite and Hermitian"):
        charge.density(skew)
    assert np.all(np.isfinite(charge.density(onsite)))
    charge.close()
    with pytest.raises(_capi.InvalidArgument, match="singular PAW compensation lattice"):
        density.CompensationCharge(context, np.zeros((3, 3)), x.positions, keys, aug, transform)
    with pytest.raises(_capi.InvalidArgument, match="radial mesh"):
        bad_aug = dict(aug, radial_grid=aug["radial_grid"][::-1].copy())
        density.CompensationCharge(context, x.lattice, x.positions, keys, bad_aug, transform)


def test_compensation_projection_matches_reference_fixture(context, golden):
    """The adjoint against the reference's project_potential_batch (host and device paths)."""
    import torch
    from conftest import relative_error
    from test_oracle_pins import _potential_on_support
    from sdft_b200 import density, synthetic
    g = golden("compensation_project_si8")
    x = synthetic.si8()
    aug = synthetic.augmentation()
    keys = synthetic.density_support(x, float(g["factor"]))
    charge = density.CompensationCharge(context, x.lattice, x.positions, keys, aug, synthetic.lm_transform(aug))
    v = _potential_on_support(keys, g["potential_keys"], g["potential"])
    out = charge.project(v)
    assert relative_error(out, g["projection"]) < 1e-12
    v_device = torch.from_numpy(v).cuda()
    torch.cuda.synchronize()
    device = charge.project(v_device)
    context.synchronize()
    assert np.array_equal(device.cpu().numpy(), out)
    charge.close()


def test_compensation_projection_is_the_adjoint_at_si64_f16(context):
    """sum_a,e P_a[e] rho_a[e] = Omega sum_G V(-G) n(G) on the config-size support
    (Si64, f = 16, ~1.5 M keys, 64 atoms), for a seeded potential and occupations."""
    from sdft_b200 import density, synthetic
    x = synthetic.si64()
    aug, rows, amplitudes, keys = _compensation_inputs(x, 128, 16.0)
    onsite = density.onsite_density(context, amplitudes, rows, np.full(128, 2.0))
    charge = density.CompensationCharge(context, x.lattice, x.positions, keys, aug, synthetic.lm_transform(aug))
    n = charge.density(onsite)
    rng = np.random.Generator(np.random.PCG64(5))
    v = rng.standard_normal(keys.shape[0]) + 1j * rng.standard_normal(keys.shape[0])
    projection = charge.project(v)
    position = {tuple(k): i for i, k in enumerate(keys.tolist())}
    v_opposite = np.array([v[position[(-h, -k, -l)]] for h, k, l in keys.tolist()])
    left = np.sum(projection * onsite)
    right = x.volume * np.sum(v_opposite * n)
    assert abs(left - right) < 1e-10 * max(abs(left), 1.0)
    charge.close()
