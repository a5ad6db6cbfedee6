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
